"""Surrogate-guided location of the gauge-Higgs transition kappa_c.

Batched HMC (one Ensemble of independent lattices, one per coupling point)
measures <L_link>, chi_link = V Var(L_link) and the plaquette; an MLP ensemble
(gauge_higgs_b200.mlp, trained on the GPU) maps (beta, kappa, lambda, 1/L) to
(<L_link>, log chi_link, plaquette); new points go where the ensemble is least
certain about the transition.  Plain HMC at every chosen point supplies the data.

The estimator uses that S_H contains -kappa B with B = 2 V D L_link, so
d<L_link>/dkappa = 2 D chi_link: the chi_link peak (the reference's transition
locator, validate_su2higgs.sh) is the inflection point of the smooth curve
<L_link>(kappa), which a smooth surrogate estimates from far fewer, noisier
points than a grid argmax of chi_link.
"""
from __future__ import annotations

import numpy as np

from . import hmc as _hmc
from .mlp import MLPEnsemble


def scan(kappas, L, ntherm=100, nmeas=300, beta=2.3, lam=0.5, nmd=12, precision="fp32", seed0=1, D=4):
    """HMC at every kappa on an L^D SU(2) + fundamental-Higgs lattice, all points in one
    batched ensemble.  Returns a dict of arrays and the number of trajectories spent."""
    kappas = np.asarray(kappas, float)
    n = len(kappas)
    ens = _hmc.Ensemble([[L] * D] * n, _hmc.FundamentalRep(2), seeds=[seed0 + i for i in range(n)], precision=precision,
                        beta=beta, kappa=kappas, lam=lam, nmd=nmd, integ="omelyan")
    ens.hot(0.8)
    ens.phi_gaussian(12345, 0.3)
    ens.run(ntherm, records=False)
    rec = ens.run(nmeas)
    ens.close()
    V = float(L ** D)
    ll = rec["L_link"]
    out = {"kappa": kappas, "L": np.full(n, L), "L_link": ll.mean(0), "L_link_err": ll.std(0) / np.sqrt(nmeas),
           "chi": V * ll.var(0), "plaq": rec["plaquette"].mean(0), "acc": rec["accepted"].mean(0)}
    return out, n * (ntherm + nmeas)


def chi_peak(kappas, chi):
    """Grid argmax of chi with a parabola through the top three points."""
    i = int(np.argmax(chi))
    if 0 < i < len(chi) - 1:
        x, y = kappas[i - 1:i + 2], chi[i - 1:i + 2]
        A = np.vstack([x * x, x, np.ones(3)]).T
        a, b, _ = np.linalg.solve(A, y)
        if a < 0:
            return float(np.clip(-b / (2 * a), x[0], x[2]))
    return float(kappas[i])


class Surrogate:
    """MLP ensemble over (beta, kappa, lambda, 1/L) -> (<L_link>, log chi, plaquette)."""

    def __init__(self, members=5, seed=11, widths=(4, 128, 128, 128, 3)):
        self.net = MLPEnsemble(widths, members, seed)
        self.xm = np.array([2.3, 0.25, 0.55, 0.125])
        self.xs = np.array([0.2, 0.1, 0.45, 0.05])

    def _x(self, beta, kappa, lam, L):
        X = np.stack(np.broadcast_arrays(beta, kappa, lam, 1.0 / np.asarray(L, float)), 1)
        return ((X - self.xm) / self.xs).astype(np.float32)

    def fit(self, pts, beta=2.3, lam=0.5, epochs=400, lr=2e-3):
        X = self._x(beta, pts["kappa"], lam, pts["L"])
        Y = np.stack([pts["L_link"], np.log(np.maximum(pts["chi"], 1e-6)), pts["plaq"]], 1)
        self.ym, self.ys = Y.mean(0), Y.std(0) + 1e-9
        Yn = ((Y - self.ym) / self.ys).astype(np.float32)
        return self.net.train(X, Yn, epochs=epochs, batch=min(32, len(X)), lr=lr)

    def predict(self, kappa, L, beta=2.3, lam=0.5):
        mean, var, per = self.net.predict(self._x(beta, kappa, lam, L), members=True)
        return per * self.ys[None, None, :] + self.ym[None, None, :]    # [members, n, 3]

    def kappa_c(self, L, lo, hi, beta=2.3, lam=0.5, h=5e-4):
        """Per member: argmax of d<L_link>/dkappa on a fine grid.  Returns the median over
        members (robust to a stray member), the spread (std) and the per-member values."""
        grid = np.arange(lo, hi + h / 2, h)
        ll = self.predict(grid, np.full(len(grid), L), beta, lam)[:, :, 0]
        dll = np.gradient(ll, grid, axis=1)
        kc = grid[np.argmax(dll, axis=1)]
        return float(np.median(kc)), float(kc.std()), kc

    def close(self):
        self.net.close()


def locate_kappa_c(L, lo=0.18, hi=0.34, n_init=5, rounds=3, per_round=4, ntherm=60, nmeas=150, beta=2.3, lam=0.5,
                   nmd=12, precision="fp32", seed=100):
    """Active learning in a shrinking trust region: a coarse grid of n_init points, then
    rounds of per_round points centred on the ensemble's kappa_c.  Round r spans
    +-max(2 spread, w0 / 2^r, 0.004), w0 = half the coarse spacing, and the next
    estimate is searched only within twice that span of the current one, so members
    that put a spurious inflection where no data lies cannot pull the estimate away.
    Returns (kappa_c, spread, trajectories, points)."""
    pts, cost = scan(np.linspace(lo, hi, n_init), L, ntherm, nmeas, beta, lam, nmd, precision, seed)
    sur = Surrogate(seed=seed)
    w0 = 0.5 * (hi - lo) / max(n_init - 1, 1)
    a, b = lo, hi
    for r in range(rounds):
        sur.fit(pts, beta, lam)
        kc, sd, per = sur.kappa_c(L, a, b, beta, lam)
        width = max(2.0 * sd, w0 / 2 ** r, 0.004)
        a, b = max(lo, kc - 2.0 * width), min(hi, kc + 2.0 * width)
        cand = np.clip(np.linspace(kc - width, kc + width, per_round), lo, hi)
        new, c = scan(cand, L, ntherm, nmeas, beta, lam, nmd, precision, seed + 97 * (r + 1))
        cost += c
        pts = {k: np.concatenate([pts[k], new[k]]) for k in pts}
    sur.fit(pts, beta, lam)
    kc, sd, _ = sur.kappa_c(L, a, b, beta, lam)
    sur.close()
    return kc, sd, cost, pts


def uniform_scan(L, lo=0.18, hi=0.34, spacing=0.005, ntherm=100, nmeas=300, beta=2.3, lam=0.5, nmd=12,
                 precision="fp32", seed=500):
    """The method without the surrogate: a uniform batched scan and the chi_link peak."""
    ks = np.arange(lo, hi + spacing / 2, spacing)
    pts, cost = scan(ks, L, ntherm, nmeas, beta, lam, nmd, precision, seed)
    return chi_peak(pts["kappa"], pts["chi"]), cost, pts
