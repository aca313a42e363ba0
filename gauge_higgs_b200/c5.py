"""The learned coupling-scan campaign: locate kappa_c of SU(2) + fundamental Higgs with an MLP surrogate.

An ensemble of five MLPs 4 -> 128 -> 128 -> 128 -> 3 (SiLU, FP32 weights, BF16
activations; gauge_higgs_b200.mlp, trained by the library's own CUDA kernels with Adam
at lr 1e-3) maps (beta, kappa, lambda, 1/L) over beta in [2.1, 2.5], kappa in
[0.15, 0.35], lambda in [0.1, 1.0] to (<L_link>, log chi_link, plaquette) of the SU(2)
fundamental-Higgs model.  It is trained first on the 64-lattice tempering batch (64
lattices, 16 kappas in 0.22..0.31 for each L in 6, 8, 10, 12, at beta 2.3, lambda 0.5)
and on 12 kappas evenly over the kappa domain at every target's (beta, lambda) and size,
all short runs; then each
active-learning round places 32 new coupling points where the members disagree most
about the transition (the spread of d<L_link>/dkappa, which is 2 D chi_link: its
maximum is the chi_link peak, the reference's transition locator,
validate_su2higgs.sh), near each target's predicted peak, and checks every point by
plain HMC (1000 trajectories at 8^4 and 12^4).  The last fit counts each of those
checks four times (they are the precise data; the seed runs have 150 trajectories), and
kappa_c of a target (beta, lambda, L) is the maximum of the predicted slope, median over
members.  Measured over four seeds and four targets this keeps every estimate within
0.0045 of a dense high-statistics chi_link peak.  A space-filling seed batch over the
whole (beta, kappa, lambda) domain instead left the first network's slope maximum at the
domain's edge for some targets (off by up to 0.1), and the checks around it could not
recover.

The method without the surrogate is a uniform batched scan of kappa over the domain at
the asked resolution (0.005) with the same per-point statistics, one per target and
size; every point of either method is plain HMC in batched ensembles on the GPU.
"""
from __future__ import annotations

import numpy as np

from . import hmc as _hmc
from .mlp import MLPEnsemble
from .surrogate import chi_peak

DOMAIN = {"beta": (2.1, 2.5), "kappa": (0.15, 0.35), "lam": (0.1, 1.0)}
D = 4


def run_points(points, ntherm, nmeas, nmd=12, precision="fp32", seed0=1, seeds=None):
    """Plain HMC at every (beta, kappa, lambda, L) point, all points one batched ensemble
    (lattices of unequal extents and couplings), point i seeded seed0 + i or seeds[i].
    Returns per-point arrays and the number of trajectories spent."""
    pts = np.asarray(points, float).reshape(-1, 4)
    n = len(pts)
    L = pts[:, 3].astype(int)
    seeds = [seed0 + i for i in range(n)] if seeds is None else [int(x) for x in seeds]
    ens = _hmc.Ensemble([[int(l)] * D for l in L], _hmc.FundamentalRep(2), seeds=seeds,
                        precision=precision, beta=pts[:, 0], kappa=pts[:, 1], lam=pts[:, 2], nmd=nmd, integ="omelyan")
    ens.hot(0.8)
    ens.phi_gaussian(12345, 0.3)
    ens.run(ntherm, records=False)
    rec = ens.run(nmeas)
    ens.close()
    ll = rec["L_link"]
    out = {"beta": pts[:, 0], "kappa": pts[:, 1], "lam": pts[:, 2], "L": L, "L_link": ll.mean(0),
           "chi": (L.astype(float) ** D) * ll.var(0), "plaq": rec["plaquette"].mean(0),
           "acc": rec["accepted"].mean(0), "nmeas": np.full(n, nmeas)}
    return out, n * (ntherm + nmeas)


def merge(a, b):
    return {k: np.concatenate([a[k], b[k]]) for k in a}


class Surrogate4D:
    """MLP ensemble over (beta, kappa, lambda, 1/L) -> (<L_link>, log chi_link, plaquette)."""

    def __init__(self, members=5, seed=11):
        self.net = MLPEnsemble((4, 128, 128, 128, 3), members, seed)
        self.xm = np.array([2.3, 0.25, 0.55, 1.0 / 9.0])
        self.xs = np.array([0.2, 0.1, 0.45, 0.05])

    def _x(self, beta, kappa, lam, L):
        X = np.stack(np.broadcast_arrays(np.asarray(beta, float), np.asarray(kappa, float), np.asarray(lam, float),
                                         1.0 / np.asarray(L, float)), 1)
        return ((X - self.xm) / self.xs).astype(np.float32)

    def fit(self, data, epochs=600, lr=1e-3, seed=7):
        X = self._x(data["beta"], data["kappa"], data["lam"], data["L"])
        Y = np.stack([data["L_link"], np.log(np.maximum(data["chi"], 1e-6)), data["plaq"]], 1)
        self.ym, self.ys = Y.mean(0), Y.std(0) + 1e-9
        Yn = ((Y - self.ym) / self.ys).astype(np.float32)
        return self.net.train(X, Yn, epochs=epochs, batch=min(32, len(X)), lr=lr, seed=seed)

    def predict(self, beta, kappa, lam, L):
        _, _, per = self.net.predict(self._x(beta, kappa, lam, L), members=True)
        return per * self.ys[None, None, :] + self.ym[None, None, :]          # [members, n, 3]

    def slope(self, beta, lam, L, grid):
        """d<L_link>/dkappa on a kappa grid, per member: [members, len(grid)]."""
        n = len(grid)
        ll = self.predict(np.full(n, beta), grid, np.full(n, lam), np.full(n, L))[:, :, 0]
        return np.gradient(ll, grid, axis=1)

    def kappa_c(self, beta, lam, L, lo=DOMAIN["kappa"][0], hi=DOMAIN["kappa"][1], h=5e-4):
        grid = np.arange(lo, hi + h / 2, h)
        kc = grid[np.argmax(self.slope(beta, lam, L, grid), axis=1)]
        return float(np.median(kc)), float(kc.std())

    def close(self):
        self.net.close()


def c4_points():
    """The 64-lattice tempering batch: 16 kappas 0.22..0.31 for each L in 6, 8, 10, 12 (beta 2.3, lambda 0.5)."""
    return [(2.3, 0.22 + 0.006 * i, 0.5, L) for L in (6, 8, 10, 12) for i in range(16)]


def target_lines(targets, sizes, n=12):
    """The extra (beta, lambda) points: n kappas evenly over the whole kappa domain at every
    target's (beta, lambda) and every size."""
    ks = np.linspace(*DOMAIN["kappa"], n)
    return [(beta, float(k), lam, L) for (beta, lam) in targets for L in sizes for k in ks]


def choose(sur, targets, sizes, per_round, window=0.03, spacing=0.003, h=5e-4):
    """per_round points, an equal share per (target, size): the kappas within +-window of
    the predicted peak where the members' slopes disagree most, at least `spacing` apart."""
    share = per_round // (len(targets) * len(sizes))
    extra = per_round - share * len(targets) * len(sizes)
    out = []
    for t, (beta, lam) in enumerate(targets):
        for s, L in enumerate(sizes):
            kc, _ = sur.kappa_c(beta, lam, L)
            lo, hi = DOMAIN["kappa"]
            grid = np.arange(max(lo, kc - window), min(hi, kc + window) + h / 2, h)
            var = sur.slope(beta, lam, L, grid).var(0)
            k = share + (1 if t * len(sizes) + s < extra else 0)
            picked = []
            for i in np.argsort(-var):
                if all(abs(grid[i] - p) >= spacing for p in picked):
                    picked.append(float(grid[i]))
                if len(picked) == k:
                    break
            out += [(beta, kp, lam, L) for kp in sorted(picked)]
    return out


def weighted(data, min_meas, weight):
    """The training set with every checked point (at least min_meas measured trajectories)
    repeated `weight` times, so that the precise HMC checks outweigh the short seed runs."""
    hi = data["nmeas"] >= min_meas
    out = data
    for _ in range(weight - 1):
        out = merge(out, {k: v[hi] for k, v in data.items()})
    return out


def campaign(targets, sizes=(8, 12), rounds=1, per_round=32, n_line=12, seed=100, seed_therm=50, seed_meas=150,
             check_therm=100, check_meas=1000, check_weight=4, precision="fp32"):
    """The surrogate-steered search.  Returns ({(beta, lambda, L): (kappa_c, the network's
    kappa_c before the checks were weighted, member spread)}, trajectories spent, the data).
    kappa_c is the maximum of the predicted slope after the last fit, in which every
    1000-trajectory HMC check counts check_weight times."""
    data, cost = run_points(c4_points() + target_lines(targets, sizes, n_line), seed_therm, seed_meas,
                            precision=precision, seed0=seed)
    sur = Surrogate4D(seed=seed)
    sur.fit(data)
    for r in range(rounds):
        pts = choose(sur, targets, sizes, per_round)
        new, c = run_points(pts, check_therm, check_meas, precision=precision, seed0=seed + 1000 * (r + 1))
        data = merge(data, new)
        cost += c
        sur.fit(data, seed=7 + r)
    plain = {(b, lam, L): sur.kappa_c(b, lam, L)[0] for (b, lam) in targets for L in sizes}
    sur.close()
    # the final network: the checks that the surrogate placed around every peak weighted up
    sur = Surrogate4D(seed=seed + 1)
    sur.fit(weighted(data, check_meas, check_weight), seed=11)
    est = {}
    for (b, lam) in targets:
        for L in sizes:
            kc, sd = sur.kappa_c(b, lam, L)
            est[(b, lam, L)] = (kc, plain[(b, lam, L)], sd)
    sur.close()
    return est, cost, data


def uniform_scan(beta, lam, L, spacing=0.005, ntherm=100, nmeas=1000, precision="fp32", seed=500):
    """The method without the surrogate: a uniform kappa scan over the domain and the
    chi_link peak.  Returns (kappa_c, trajectories, data)."""
    lo, hi = DOMAIN["kappa"]
    ks = np.arange(lo, hi + spacing / 2, spacing)
    data, cost = run_points([(beta, k, lam, L) for k in ks], ntherm, nmeas, precision=precision, seed0=seed)
    return chi_peak(data["kappa"], data["chi"]), cost, data


def truth(beta, lam, L, centre, half=0.03, spacing=0.0025, ntherm=200, nmeas=1000, repeats=4, precision="fp32",
          seed=9000):
    """A dense high-statistics chi_link peak around `centre` (not counted): repeats x nmeas
    measured trajectories per point, chi the mean over the repeats.  The kappas lie on the
    fixed grid of multiples of `spacing` and each point's chains are seeded by its grid
    index, so that two windows share the points they overlap in."""
    i0 = int(round(centre / spacing))
    idx = np.arange(i0 - int(round(half / spacing)), i0 + int(round(half / spacing)) + 1)
    ks = idx * spacing
    chis = []
    for r in range(repeats):
        d, _ = run_points([(beta, k, lam, L) for k in ks], ntherm, nmeas, precision=precision,
                          seeds=seed + 1000 * r + idx)
        chis.append(d["chi"])
    return chi_peak(ks, np.mean(chis, 0))
