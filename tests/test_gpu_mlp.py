"""GPU MLP ensemble (the coupling-scan surrogate) against its FP64 restatement
(oracle/mlp_oracle.py): forward, gradients, one Adam step, and training."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, size=(n, 4)).astype(np.float32)
    y = np.stack([np.sin(2 * x[:, 0]) + x[:, 1], x[:, 2] * x[:, 3], np.cos(x[:, 0] + x[:, 3])], 1).astype(np.float32)
    return x, y


def test_forward_and_gradients_match_oracle():
    from gauge_higgs_b200.mlp import MLPEnsemble
    from oracle import mlp_oracle as mo
    net = MLPEnsemble(members=3, seed=5)
    x, y = data(100)
    p = net.params()
    g, loss = net.grad(x, y)
    mean, var, per = net.predict(x, members=True)
    for m in range(3):
        out, _, _ = mo.forward(p[m], net.widths, x)
        assert np.abs(per[m] - out).max() < 2e-3 * max(1.0, np.abs(out).max())
        lo, go = mo.loss_and_grad(p[m], net.widths, x, y)
        assert abs(loss[m] - lo) < 1e-3 * lo
        assert np.abs(g[m] - go).max() < 1e-2 * np.abs(go).max()
        # per-layer relative agreement of the weight gradients
        for (w0, w1, shape), (b0, b1) in net.layout():
            a, b = g[m][w0:w1], go[w0:w1]
            assert np.linalg.norm(a - b) < 2e-2 * np.linalg.norm(b) + 1e-9
    assert np.allclose(mean, per.mean(0), atol=1e-6) and np.allclose(var, per.var(0), atol=1e-6)
    net.close()


def test_adam_step_matches_oracle():
    from gauge_higgs_b200.mlp import MLPEnsemble
    from oracle import mlp_oracle as mo
    net = MLPEnsemble(members=2, seed=9)
    x, y = data(64, 1)
    p0 = net.params().astype(np.float64)
    g, _ = net.grad(x, y)
    net.adam_step(1e-3)
    p1 = net.params()
    for m in range(2):
        pe, _, _ = mo.adam(p0[m], g[m].astype(np.float64), 0.0, 0.0, 1, 1e-3)
        assert np.abs(p1[m] - pe).max() < 1e-6
    net.close()


def test_training_reduces_loss_and_members_differ():
    from gauge_higgs_b200.mlp import MLPEnsemble
    net = MLPEnsemble(members=5, seed=3)
    x, y = data(512, 2)
    _, l0 = net.grad(x, y)
    loss = net.train(x, y, epochs=150, batch=64, lr=2e-3)
    assert np.all(loss < 0.1 * l0), (loss, l0)
    xt, yt = data(200, 7)
    mean, var = net.predict(xt)
    assert np.mean((mean - yt) ** 2) < 0.02
    assert np.all(var.mean(0) > 0)
    net.close()
