"""Pins the MLP restatement (oracle/mlp_oracle.py) by finite differences: the
reference has no learned component, so the gradient of the restatement is checked
against the derivative of its own loss (without BF16 rounding, which is not
differentiable)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_gradient_finite_difference():
    rng = np.random.default_rng(0)
    widths = [4, 16, 16, 3]
    P = sum(a * b + b for a, b in zip(widths[:-1], widths[1:]))
    p = rng.normal(scale=0.4, size=P)
    x = rng.uniform(-1, 1, size=(20, 4))
    y = rng.normal(size=(20, 3))
    _, g = mo.loss_and_grad(p, widths, x, y, round_bf16=False)
    h = 1e-6
    for k in rng.choice(P, 40, replace=False):
        e = np.zeros(P)
        e[k] = h
        fd = (mo.loss_and_grad(p + e, widths, x, y, False)[0] - mo.loss_and_grad(p - e, widths, x, y, False)[0]) / (2 * h)
        assert abs(fd - g[k]) < 1e-7 + 1e-5 * abs(fd)


def test_bf16_rounding():
    # 1 + 2^-8 and 1 + 3*2^-8 are midpoints of BF16 neighbours: ties go to the even mantissa
    v = np.array([1.0, 1.00390625, 1.01171875, 1.001953125, -3.14159, 0.0], np.float32)
    r = mo.bf16(v)
    assert list(r[:4]) == [1.0, 1.0, 1.015625, 1.0]
    assert abs(r[4] + 3.140625) < 1e-7 and r[5] == 0.0
