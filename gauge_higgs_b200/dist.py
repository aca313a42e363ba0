"""Replica tempering across the ranks of a process group (one GPU per rank).

The lattices of a ladder are spread over the ranks; each rank evolves its share as
one Ensemble (every trajectory one CUDA graph launch).  A swap exchanges coupling
labels, not fields (the mechanism of src/hmc/replica_tempering.hpp:157-205 with the
labels moving instead of (U, phi), as the device pass does), so after each swap
interval only three numbers per lattice cross between ranks -- its coupling, its
B and its extents key -- in one all_gather.  Every rank then replays the same swap
pass and relabels its own lattices, so all ranks agree on every decision without a
further exchange.  On one rank the decisions are exactly those of the device pass
of a single Ensemble (gh_temper_enable).
"""
from __future__ import annotations

import math

import numpy as np

from ._lib import LIB
from .hmc import Ensemble

SWAP_STREAM = 0x57A9


def swap_energy(coupling, plaquette, L_link, volume, D):
    """B of the tempered coupling: beta -> n_plaq (plaquette - 1) (S_g = -beta B + const);
    kappa -> 2 V D L_link (S_H = ... - kappa B)."""
    if coupling == "beta":
        return volume * (D * (D - 1) // 2) * (np.asarray(plaquette, float) - 1.0)
    return 2.0 * np.asarray(L_link, float) * volume * D


def temper_pass(c, B, groups, counter, seed, stats=None):
    """One even + odd swap pass (src/hmc/replica_tempering.hpp:157-167,170-190) over the
    ladders `groups` (lists of lattice indices with equal extents, groups in the order
    of their extents, as the device pass); c, B: coupling and energy of every lattice.
    Pairs (k, k+1) of a ladder sorted by c propose a label exchange with
    Delta = (c_i - c_j)(B_i - B_j), accepted if Delta <= 0 or uniform(seed,
    key(0x57A9, counter)) < exp(-Delta), the counter advancing at every proposal.
    Returns the new couplings and the counter; stats (optional dict pair -> [attempts,
    accepts]) is updated with pairs numbered along the ladders."""
    c = np.array(c, dtype=float, copy=True)
    pid0 = 0
    for g in groups:
        order = sorted(g, key=lambda l: c[l])
        for start in (0, 1):
            for k in range(start, len(order) - 1, 2):
                li, lj = order[k], order[k + 1]
                delta = (c[li] - c[lj]) * (B[li] - B[lj])
                counter += 1
                ok = delta <= 0.0 or LIB.gh_rng_uniform(seed, LIB.gh_rng_key(SWAP_STREAM, counter, 0, 0, 0)) < math.exp(-delta)
                if stats is not None:
                    a = stats.setdefault(pid0 + k, [0, 0])
                    a[0] += 1
                    a[1] += int(ok)
                if ok:
                    c[li], c[lj] = c[lj], c[li]
                    order[k], order[k + 1] = lj, li
        pid0 += len(order) - 1
    return c, counter


def ladders(extents):
    """Groups of equal-extent lattices, in the lexicographic order of the extents."""
    by = {}
    for i, e in enumerate(extents):
        by.setdefault(tuple(e), []).append(i)
    return [by[k] for k in sorted(by)]


def exchange(mine, values, n_total, group=None):
    """all_gather of per-lattice rows: mine (global indices of this rank's lattices),
    values [len(mine), m]; returns [n_total, m] on every rank."""
    import torch.distributed as dist
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, (list(map(int, mine)), np.asarray(values, float).tolist()), group=group)
    out = np.zeros((n_total, np.asarray(values).shape[1]))
    for idx, rows in parts:
        if idx:
            out[idx] = np.asarray(rows, float)
    return out


class ShardedEnsemble:
    """An ensemble of lattices spread over the ranks of the default process group (or
    `group`), with replica tempering in beta or kappa across all of them.

    extents, seeds, beta, kappa, lam: per lattice, over the whole ensemble; rank r
    holds the r-th contiguous share.  temper: "beta", "kappa" or None; n_sweep:
    trajectories between swap passes (ReplicaTempering::n_sweep)."""

    def __init__(self, extents, rep, seeds, beta, kappa, lam, temper="beta", swap_seed=0x5A7AB1EC, n_sweep=1,
                 group=None, **kw):
        import torch.distributed as dist
        self.group = group
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        n = len(extents)
        if n < self.world:
            raise ValueError("fewer lattices than ranks")
        self.n = n
        self.extents = [list(e) for e in extents]
        self.mine = np.array_split(np.arange(n), self.world)[self.rank]
        b = np.broadcast_to(np.asarray(beta, float), (n,))
        k = np.broadcast_to(np.asarray(kappa, float), (n,))
        self.lam = np.broadcast_to(np.asarray(lam, float), (n,)).copy()
        self.ens = Ensemble([self.extents[i] for i in self.mine], rep, seeds=[seeds[i] for i in self.mine],
                            beta=b[self.mine], kappa=k[self.mine], lam=self.lam[self.mine], **kw)
        self.D = self.ens.D
        self.temper, self.swap_seed, self.n_sweep = temper, int(swap_seed), int(n_sweep)
        self.groups = ladders(self.extents)
        self.counter = 0
        self.traj = 0
        self.stats = {}
        if temper is not None:
            c = b if temper == "beta" else k
            for g in self.groups:
                cs = sorted(c[i] for i in g)
                if any(not (y > x) for x, y in zip(cs, cs[1:])):
                    raise ValueError("the tempered coupling of equal-extent lattices must be strictly increasing")

    def __getattr__(self, name):          # hot, phi_gaussian, records, ... of the local Ensemble
        return getattr(self.ens, name)

    def run(self, ntraj):
        """ntraj trajectories of every lattice; returns this rank's records [ntraj, n_local]."""
        out = []
        for _ in range(int(ntraj)):
            rec = self.ens.run(1)[0]
            self.traj += 1
            if self.temper is not None and self.traj % self.n_sweep == 0:
                self._swap(rec)
            out.append(rec)
        return np.stack(out)

    def _swap(self, rec):
        vol = np.array([np.prod(self.extents[i]) for i in self.mine], float)
        c = rec["beta"] if self.temper == "beta" else rec["kappa"]
        B = swap_energy(self.temper, rec["plaquette"], rec["L_link"], vol, self.D)
        allv = exchange(self.mine, np.stack([c, B], 1), self.n, self.group)
        cnew, self.counter = temper_pass(allv[:, 0], allv[:, 1], self.groups, self.counter, self.swap_seed,
                                         self.stats)
        for j, i in enumerate(self.mine):
            if cnew[i] != allv[i, 0]:
                bj, kj, lj = self.ens.couplings(j)
                if self.temper == "beta":
                    bj = cnew[i]
                else:
                    kj = cnew[i]
                self.ens.set_couplings(j, bj, kj, lj)
