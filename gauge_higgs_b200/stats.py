"""Time-series statistics of the measurement loop (host side).

The quantities of src/measure/observables.hpp:104-145, written from their
definitions: mean, population variance, susceptibility chi = V * Var, Binder
cumulant U4 = 1 - <d^4> / (3 <d^2>^2) (centred on the mean), and the jackknife
error of the mean over 16 contiguous bins.  The bin rule is the reference's (it
fixes the printed error bars): bins of floor(n / nbins) samples from the start,
nbins lowered to max(2, n // 2) for a series shorter than 2 nbins, no error for
n < 2.
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

    def central_moment(self, k):
        """k-th moment about the sample mean, 1/n normalisation."""
        if not self.x:
            return 0.0
        m = self.mean()
        return sum((v - m) ** k for v in self.x) / len(self.x)

    def var(self):
        return self.central_moment(2)

    def susceptibility(self, volume):
        return volume * self.var()

    def binder(self):
        m2 = self.central_moment(2)
        return 1.0 - self.central_moment(4) / (3.0 * m2 * m2) if m2 > 0.0 else 0.0

    def binned_error(self, nbins=16):
        """Jackknife error of the mean over contiguous bins (leave one bin out)."""
        total = self.n()
        if total < 2:
            return 0.0
        nb = max(2, total // 2) if total < 2 * nbins else nbins
        width = total // nb
        sums = [sum(self.x[b * width:(b + 1) * width]) for b in range(nb)]
        allsum = sum(sums)
        theta = [(allsum - sb) / ((nb - 1) * width) for sb in sums]
        tbar = sum(theta) / nb
        return math.sqrt((nb - 1) / nb * sum((t - tbar) ** 2 for t in theta))
