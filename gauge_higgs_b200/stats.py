"""Time-series statistics of the measurement loop (host side).

Stats restates src/measure/observables.hpp:104-145: mean, population variance,
susceptibility chi = V * Var, Binder cumulant U4 = 1 - <d^4> / (3 <d^2>^2)
(centred on the mean), and the block-jackknife error of the mean with 16 bins.
"""
from __future__ import annotations

import math


class Stats:
    def __init__(self, values=None):
        self.x = list(values) if values is not None else []

    def add(self, v):
        self.x.append(float(v))

    def n(self):
        return len(self.x)

    def mean(self):
        return sum(self.x) / len(self.x) if self.x else 0.0

    def var(self):
        if not self.x:
            return 0.0
        m = self.mean()
        return sum(v * v for v in self.x) / len(self.x) - m * m

    def susceptibility(self, volume):
        return volume * self.var()

    def binder(self):
        if not self.x:
            return 0.0
        m = self.mean()
        m2 = sum((v - m) ** 2 for v in self.x) / len(self.x)
        m4 = sum((v - m) ** 4 for v in self.x) / len(self.x)
        return 1.0 - m4 / (3.0 * m2 * m2) if m2 > 0.0 else 0.0

    def binned_error(self, nbins=16):
        N = self.n()
        if N < 2 * nbins:
            nbins = max(2, N // 2)
        if N < 2:
            return 0.0
        bs = N // nbins
        bm = [sum(self.x[b * bs:(b + 1) * bs]) / bs for b in range(nbins)]
        mb = sum(bm) / len(bm)
        v = sum((b - mb) ** 2 for b in bm) / (len(bm) - 1)
        return math.sqrt(v / len(bm))
