"""FP64 numpy restatement of the surrogate MLP (TEST INFRASTRUCTURE ONLY).

Same network and loss as gauge_higgs_b200/csrc/gh_mlp.cu: SiLU between layers,
hidden activations rounded to BF16 where the GPU stores them, mean squared
error, Adam (beta1 0.9, beta2 0.999, eps 1e-8).  Used to check the GPU
gradients and one optimiser step.  The reference has no learned component, so
this part of the parity is against this restatement only (parity unpinned by
the reference).
"""
import numpy as np


def bf16(x):
    """Round FP32 values to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((f + 0x7FFF + ((f >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(p, widths):
    Ws, bs, off = [], [], 0
    for a, b in zip(widths[:-1], widths[1:]):
        Ws.append(p[off:off + a * b].reshape(b, a).astype(np.float64))
        off += a * b
        bs.append(p[off:off + b].astype(np.float64))
        off += b
    return Ws, bs


def forward(p, widths, x, round_bf16=True):
    Ws, bs = unpack(p, widths)
    a = np.asarray(x, np.float64)
    zs, acts = [], [a]
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = a @ W.T + b
        zs.append(z)
        if l < len(Ws) - 1:
            a = bf16(silu(z)) if round_bf16 else silu(z)
            acts.append(a)
        else:
            a = z
    return a, zs, acts


def loss_and_grad(p, widths, x, y, round_bf16=True):
    Ws, bs = unpack(p, widths)
    out, zs, acts = forward(p, widths, x, round_bf16)
    B, k = out.shape
    d = out - y
    loss = float(np.mean(d * d))
    g = 2.0 * d / (B * k)
    grads = []
    for l in range(len(Ws) - 1, -1, -1):
        gW = g.T @ acts[l]
        gb = g.sum(0)
        grads.append((gW, gb))
        if l > 0:
            g = (g @ Ws[l]) * dsilu(zs[l - 1])
    grads.reverse()
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat


def adam(p, g, m1, m2, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    p = p - lr * (m1 / (1 - b1 ** t)) / (np.sqrt(m2 / (1 - b2 ** t)) + eps)
    return p, m1, m2
