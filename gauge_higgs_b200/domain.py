"""Domain decomposition of one lattice over several GPUs (the reference's src/mpi/:
DistLattice, halo_exchange_raw, DistGaugeHMC / DistGaugeHiggsHMC in
src/mpi/gauge_mpi.hpp:26-290 and src/mpi/higgs_mpi.hpp:150-226).

The global lattice G is split over a process grid P (dimension 0 fastest, as the
site numbering); a rank's subdomain is stored padded by one halo layer on each side
of every split direction and whole in the others, and its context is told the
interior box and global offset (gh_set_domain), so that kernels touch the interior
only and the counter RNG is keyed on global site indices: hot starts, scalar
initialisation and momentum heatbaths are the whole lattice's draws, and a decomposed
run reproduces the single-GPU run.  Halos are exchanged by whole planes, direction
after direction (filling edges and corners), before every force and action
evaluation; H is summed over ranks in rank order and every rank takes the same
accept decision from the same key.

Transports: InProcessTransport (several subdomains of one process, e.g. on one GPU;
the kernels of one subdomain never wait for another's) and TorchTransport (one
subdomain per rank over a torch.distributed group: NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

import math

import numpy as np


def _rank_of(coords, P):
    r, m = 0, 1
    for c, p in zip(coords, P):
        r += c * m
        m *= p
    return r


def _coords_of(rank, P):
    c = []
    for p in P:
        c.append(rank % p)
        rank //= p
    return c


class Subdomain:
    """Geometry of one rank's piece of a G lattice split over the process grid P."""

    def __init__(self, G, P, coords):
        self.G = [int(g) for g in G]
        self.P = [int(p) for p in P]
        self.D = len(self.G)
        if len(self.P) != self.D or any(g % p for g, p in zip(self.G, self.P)):
            raise ValueError("the process grid must have D entries that divide the global extents")
        self.coords = [int(c) for c in coords]
        self.rank = _rank_of(self.coords, self.P)
        self.split = [p > 1 for p in self.P]
        self.Lloc = [g // p for g, p in zip(self.G, self.P)]
        self.L = [l + 2 if s else g for l, s, g in zip(self.Lloc, self.split, self.G)]     # stored extents
        self.lo = [1 if s else 0 for s in self.split]
        self.hi = [l + 1 if s else g for l, s, g in zip(self.Lloc, self.split, self.G)]
        self.goff = [c * l if s else 0 for c, l, s in zip(self.coords, self.Lloc, self.split)]
        self.split_dirs = [mu for mu in range(self.D) if self.split[mu]]
        self.strides = [int(np.prod(self.L[:mu])) for mu in range(self.D)]
        self.V = int(np.prod(self.L))
        self.V_interior = int(np.prod([h - l for l, h in zip(self.lo, self.hi)]))

    def neighbour_rank(self, nu, step):
        c = list(self.coords)
        c[nu] = (c[nu] + step) % self.P[nu]
        return _rank_of(c, self.P)

    def plane_sites(self, nu, layer):
        """Local sites with x_nu = layer, in the order of the device's halo buffers
        (mixed radix over the other directions, direction 0 fastest)."""
        others = [mu for mu in range(self.D) if mu != nu]
        grids = np.meshgrid(*[np.arange(self.L[mu]) for mu in reversed(others)], indexing="ij")
        s = np.full(grids[0].shape if grids else (1,), layer * self.strides[nu], np.int64)
        for g, mu in zip(grids, reversed(others)):
            s = s + g * self.strides[mu]
        return s.reshape(-1)

    def coords_of_site(self, s):
        s = np.asarray(s, np.int64)
        return [(s // self.strides[mu]) % self.L[mu] for mu in range(self.D)]

    def interior_sites(self):
        """Local interior sites (site order) and their global site indices."""
        x = self.coords_of_site(np.arange(self.V))
        inside = np.ones(self.V, bool)
        for mu in range(self.D):
            inside &= (x[mu] >= self.lo[mu]) & (x[mu] < self.hi[mu])
        s = np.nonzero(inside)[0]
        return s, self.global_site(s)

    def global_site(self, s):
        """Global site index of local sites s (wrapping halo sites periodically)."""
        x = self.coords_of_site(s)
        g, m = 0, 1
        for mu in range(self.D):
            gx = (x[mu] - self.lo[mu] + self.goff[mu]) % self.G[mu]
            g = g + gx * m
            m *= self.G[mu]
        return g


def halo_exchange(parts, transport, pack, unpack):
    """Width-1 halo of every split direction, one direction after the other
    (src/mpi/gauge_mpi.hpp:101-139): the last interior layer goes to the +nu
    neighbour's lower halo, the first interior layer to the -nu neighbour's upper halo.
    parts: the local Subdomains; pack(i, nu, layer) -> buffer of part i's plane;
    unpack(i, nu, layer, buffer)."""
    if not parts:
        return
    for nu in parts[0].split_dirs:
        recv = transport.shift([pack(i, nu, p.hi[nu] - 1) for i, p in enumerate(parts)], nu, +1)
        for i, p in enumerate(parts):
            unpack(i, nu, 0, recv[i])
        recv = transport.shift([pack(i, nu, p.lo[nu]) for i, p in enumerate(parts)], nu, -1)
        for i, p in enumerate(parts):
            unpack(i, nu, p.hi[nu], recv[i])


class InProcessTransport:
    """All subdomains of the grid in this process (part i is rank i)."""

    def __init__(self, G, P):
        self.P = list(P)
        self.nranks = int(np.prod(self.P))
        self.parts = [Subdomain(G, P, _coords_of(r, self.P)) for r in range(self.nranks)]

    def local_parts(self):
        return self.parts

    def shift(self, bufs, nu, step):
        # part i receives what its -step neighbour sent
        return [bufs[p.neighbour_rank(nu, -step)] for p in self.parts]

    def sum(self, values):
        t = 0.0
        for v in values:            # rank order: the same sum on every rank and every run
            t += float(v)
        return t


class TorchTransport:
    """One subdomain per rank of a torch.distributed group (NCCL for device buffers,
    gloo for CPU tensors).  Reductions gather every rank's value and add them in rank
    order, so all ranks hold the same bits."""

    def __init__(self, G, P, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.P = list(P)
        self.nranks = int(np.prod(self.P))
        ws = dist.get_world_size(group)
        if ws != self.nranks:
            raise ValueError(f"process grid {P} needs {self.nranks} ranks, the group has {ws}")
        self.rank = dist.get_rank(group)
        self.parts = [Subdomain(G, P, _coords_of(self.rank, self.P))]

    def local_parts(self):
        return self.parts

    def shift(self, bufs, nu, step):
        import torch
        p = self.parts[0]
        send = bufs[0]
        recv = torch.empty_like(send)
        dst, src = p.neighbour_rank(nu, step), p.neighbour_rank(nu, -step)
        ops = [self.dist.P2POp(self.dist.isend, send, dst, self.group),
               self.dist.P2POp(self.dist.irecv, recv, src, self.group)]
        for r in self.dist.batch_isend_irecv(ops):
            r.wait()
        if recv.is_cuda:                    # the plane has landed before a context's stream reads it
            torch.cuda.current_stream().synchronize()
        return [recv]

    def sum(self, values):
        import torch
        v = torch.tensor([float(values[0])], dtype=torch.float64)
        if self.dist.get_backend(self.group) == "nccl":
            v = v.cuda()
        out = [torch.empty_like(v) for _ in range(self.nranks)]
        self.dist.all_gather(out, v, group=self.group)
        t = 0.0
        for x in out:
            t += float(x.item())
        return t


OMELYAN_LAMBDA = 0.1931833275037836


class DomainHMC:
    """Domain-decomposed gauge (+ Higgs) HMC on the GPU, the counterpart of the
    reference's DistGaugeHMC / DistGaugeHiggsHMC (src/mpi/gauge_mpi.hpp:208-287,
    src/mpi/higgs_mpi.hpp:150-226): one context per local subdomain, halos refreshed
    before every force and action, dH and the accept decision global.  rep None: pure
    gauge (keys 0xA1 / 0xB2), otherwise gauge + Higgs (0xC3, 0xD4 / 0xE5).

    transport: InProcessTransport (all subdomains here) or TorchTransport (this
    rank's).  Results do not depend on the process grid: fields evolve bit for bit as
    on one GPU, and dH differs only by the order of the global sums."""

    def __init__(self, G, transport, rep=None, N=None, seed=1, precision="fp64", beta=2.3, kappa=0.1, lam=0.5,
                 tau=1.0, nmd=20, integ="omelyan"):
        import ctypes as C
        import torch
        from . import hmc as _hmc
        from ._lib import LIB, check
        self._C, self._LIB, self._check, self._torch = C, LIB, check, torch
        self.G = list(G)
        self.D = len(self.G)
        self.transport = transport
        self.parts = transport.local_parts()
        self.rep = rep
        self.pure = rep is None
        self.seed = int(seed)
        self.tau, self.nmd, self.integ = float(tau), int(nmd), integ
        self.traj_count = 0
        self.accept_count = 0
        self.last_dH = 0.0
        self.h = []
        for p in self.parts:
            if self.pure:
                h = _hmc.GaugeHMC(p.L, N, seed=seed, precision=precision, beta=beta, nmd=nmd, tau=tau, integ=integ)
            else:
                h = _hmc.GaugeHiggsHMC(p.L, rep, seed=seed, precision=precision, beta=beta, kappa=kappa, lam=lam,
                                       nmd=nmd, tau=tau, integ=integ)
            ia = lambda v: (C.c_int * self.D)(*v)
            check(LIB.gh_set_domain(h.ctx.h, 0, ia(self.G), ia(p.lo), ia(p.hi), ia(p.goff)), h.ctx.h)
            self.h.append(h)
        self.N = self.h[0].N
        self._bufs = {}
        self._dirty = True

    # ---- halos ----
    def _buf(self, i, field, nu):
        key = (i, field, nu)
        if key not in self._bufs:
            n = self._C.c_longlong()
            self._check(self._LIB.gh_halo_count(self.h[i].ctx.h, 0, field, nu, self._C.byref(n)), self.h[i].ctx.h)
            dt = self._torch.float64 if self.h[i].precision == "fp64" else self._torch.float32
            self._bufs[key] = (n.value, dt)
        n, dt = self._bufs[key]
        return self._torch.empty(2 * n, dtype=dt, device="cuda")

    def exchange(self):
        fields = [0] if self.pure else [0, 1]
        for field in fields:
            def pack(i, nu, layer):
                b = self._buf(i, field, nu)
                self._check(self._LIB.gh_halo_pack(self.h[i].ctx.h, 0, field, nu, layer, b.data_ptr()), self.h[i].ctx.h)
                self.h[i].sync()            # the plane is complete before anyone else reads the buffer
                return b

            def unpack(i, nu, layer, b):
                self._check(self._LIB.gh_halo_unpack(self.h[i].ctx.h, 0, field, nu, layer, b.data_ptr()),
                            self.h[i].ctx.h)
            # the contexts' own streams: their work on the fields is done before the planes are read
            for h in self.h:
                h.sync()
            halo_exchange(self.parts, self.transport, pack, unpack)
        for h in self.h:
            h.sync()
        self._dirty = False

    def _fresh(self):
        if self._dirty:
            self.exchange()

    # ---- initialisation (global-index keys: the whole lattice's draws) ----
    def hot(self, sigma=0.8):
        for h in self.h:
            h.hot(sigma)
        self._dirty = True

    def cold(self):
        for h in self.h:
            h.cold()
        self._dirty = True

    def phi_gaussian(self, stream=12345, sigma=0.3):
        for h in self.h:
            h.phi_gaussian(stream, sigma)
        self._dirty = True

    # ---- MD ----
    def kick(self, eps):
        self._fresh()
        for h in self.h:
            h.kick(eps)

    def drift(self, eps):
        for h in self.h:
            h.drift(eps)
        self._dirty = True

    def md_evolve(self):
        """The reference's leapfrog / Omelyan 2MN sequences (src/mpi/higgs_mpi.hpp:198-208)."""
        eps = self.tau / self.nmd
        if self.integ == "leapfrog":
            self.kick(0.5 * eps)
            for i in range(self.nmd):
                self.drift(eps)
                if i != self.nmd - 1:
                    self.kick(eps)
            self.kick(0.5 * eps)
        else:
            lam = OMELYAN_LAMBDA
            self.kick(lam * eps)
            for i in range(self.nmd):
                self.drift(0.5 * eps)
                self.kick((1.0 - 2.0 * lam) * eps)
                self.drift(0.5 * eps)
                self.kick((2.0 * lam if i != self.nmd - 1 else lam) * eps)

    # ---- global measurements ----
    def measure_parts(self):
        self._fresh()
        return [h.measure() for h in self.h]

    def hamiltonian(self):
        return self.transport.sum([m["H"] for m in self.measure_parts()])

    def measure(self):
        """Global plaquette, L_link, L_phi (interior averages weighted by volume) and H."""
        ms = self.measure_parts()
        Vg = float(np.prod(self.G))
        out = {"H": self.transport.sum([m["H"] for m in ms])}
        for k in ("plaquette", "L_link", "L_phi"):
            out[k] = self.transport.sum([m[k] * p.V_interior for m, p in zip(ms, self.parts)]) / Vg
        return out

    def trajectory(self):
        """src/mpi/higgs_mpi.hpp:210-225 (src/mpi/gauge_mpi.hpp:270-285 for pure gauge)."""
        from ._lib import LIB
        for h in self.h:
            h.set_traj_count(0, self.traj_count, self.accept_count)
            h.refresh_momenta()
            self._check(LIB.gh_save_fields(h.ctx.h), h.ctx.h)
        self._dirty = True
        Hi = self.hamiltonian()
        self.md_evolve()
        if self.h[0].precision == "fp64":
            # the reference's end-of-trajectory reunitarisation; FP32-MD projects in every drift
            for h in self.h:
                h.reunitarize_all()
        self._dirty = True
        Hf = self.hamiltonian()
        self.last_dH = Hf - Hi
        self.traj_count += 1
        key = LIB.gh_rng_key(0xB2 if self.pure else 0xE5, self.traj_count, 0, 0, 0)
        r = LIB.gh_rng_uniform(self.seed, key)
        acc = bool(self.last_dH <= 0.0 or r < math.exp(-self.last_dH))
        if acc:
            self.accept_count += 1
        else:
            for h in self.h:
                self._check(LIB.gh_restore_fields(h.ctx.h), h.ctx.h)
            self._dirty = True
        return acc

    def acceptance(self):
        return self.accept_count / self.traj_count if self.traj_count else 0.0

    def close(self):
        for h in self.h:
            h.close()
        self.h = []
