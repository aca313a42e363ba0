"""Host binding of the GPU MLP ensemble (gh_mlp_* in include/gauge_higgs_b200.h).

Training, gradients and prediction run in the library's own CUDA kernels
(gauge_higgs_b200/csrc/gh_mlp.cu); this class only moves FP32 arrays."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import LIB, GaugeHiggsError


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check(rc):
    if rc != 0:
        raise GaugeHiggsError(rc, (LIB.gh_mlp_last_error() or b"").decode())


class MLPEnsemble:
    def __init__(self, widths=(4, 128, 128, 128, 3), members=5, seed=1):
        self.widths = list(widths)
        self.members = members
        w = (C.c_int * len(widths))(*widths)
        h = C.c_void_p()
        _check(LIB.gh_mlp_create(members, w, len(widths) - 1, seed, C.byref(h)))
        self.h = h
        p = C.c_long()
        _check(LIB.gh_mlp_num_params(self.h, C.byref(p)))
        self.P = p.value

    def close(self):
        if self.h:
            LIB.gh_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.zeros((self.members, self.P), np.float32)
        _check(LIB.gh_mlp_get_params(self.h, _f(out)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(LIB.gh_mlp_set_params(self.h, _f(p)))

    def grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros((self.members, self.P), np.float32)
        loss = np.zeros(self.members, np.float32)
        _check(LIB.gh_mlp_grad(self.h, _f(x), _f(y), len(x), _f(g), _f(loss)))
        return g, loss

    def adam_step(self, lr):
        _check(LIB.gh_mlp_adam_step(self.h, C.c_float(lr)))

    def train(self, x, y, epochs=200, batch=64, lr=1e-3, seed=7):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = np.zeros(self.members, np.float32)
        _check(LIB.gh_mlp_train(self.h, _f(x), _f(y), len(x), epochs, batch, C.c_float(lr), seed, _f(loss)))
        return loss

    def predict(self, x, members=False):
        x = np.ascontiguousarray(x, np.float32)
        n, k = len(x), self.widths[-1]
        mean = np.zeros((n, k), np.float32)
        var = np.zeros((n, k), np.float32)
        per = np.zeros((self.members, n, k), np.float32) if members else None
        _check(LIB.gh_mlp_predict(self.h, _f(x), n, _f(per) if members else None, _f(mean), _f(var)))
        return (mean, var, per) if members else (mean, var)

    def layout(self):
        """(W, b) slices of one member's parameter vector, layer by layer (W is [out][in])."""
        out, off = [], 0
        for a, b in zip(self.widths[:-1], self.widths[1:]):
            out.append(((off, off + a * b, (b, a)), (off + a * b, off + a * b + b)))
            off += a * b + b
        return out
