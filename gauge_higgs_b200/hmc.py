"""Host-side mirror of the reference's HMC interface over the B200 engine.

Class and method names follow the reference (hlammiv/gauge_higgs):
  FundamentalRep / AdjointRep / GeneralRep      src/rep/rep_fundamental.hpp, rep_adjoint.hpp, rep_general.hpp
  GaugeHiggsHMC (kick, drift, md_evolve, hamiltonian, refresh_momenta, trajectory)
                                                src/hmc/gauge_higgs_hmc.hpp:15-195
  GaugeHMC (pure gauge)                         src/hmc/hmc.hpp:12-96
  Ensemble: many lattices in one context, with replica tempering in kappa
                                                mechanism of src/hmc/replica_tempering.hpp:77-219
Fields cross the boundary as numpy arrays in the reference's layouts:
  U [V, D, N, N] complex128, P [V, D, N^2-1] float64, phi / pi [V, d] complex128.
All compute runs in libgauge_higgs_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
import numpy as np

from . import _lib
from ._lib import LIB, check, GaugeHiggsError, RepDesc, Obs, TrajRecord, TRAJ_DTYPE

LEAPFROG, OMELYAN = _lib.LEAPFROG, _lib.OMELYAN
_INTEG = {"leapfrog": LEAPFROG, "omelyan": OMELYAN, LEAPFROG: LEAPFROG, OMELYAN: OMELYAN}
# "fp32" / "fp32-md": FP32 fields and forces, the drift's exp(i eps P), product and
# SU(N) projection in FP64; "fp32-all": those in FP32 as well (non-default variant)
_PREC = {"fp64": _lib.PREC_FP64, "fp32": _lib.PREC_FP32_MD, "fp32-md": _lib.PREC_FP32_MD,
         "fp32-all": _lib.PREC_FP32_ALL, _lib.PREC_FP64: _lib.PREC_FP64, _lib.PREC_FP32_MD: _lib.PREC_FP32_MD,
         _lib.PREC_FP32_ALL: _lib.PREC_FP32_ALL}


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ---------------------------------------------------------------------------
# Representations (src/rep/representation.hpp:12-32)
# ---------------------------------------------------------------------------
class Representation:
    kind = _lib.REP_NONE
    real = False
    n_boxes = 0
    dimT = 0
    T = None
    W = None

    def __init__(self, N, d):
        self.N, self.d = N, d

    def desc(self):
        self._keep = []
        r = RepDesc()
        r.kind, r.d, r.real, r.n_boxes, r.dimT = self.kind, self.d, int(self.real), self.n_boxes, self.dimT
        for name in ("T", "W"):
            a = getattr(self, name)
            if a is not None:
                a = np.ascontiguousarray(a, np.complex128).view(np.float64)
                self._keep.append(a)
                setattr(r, name, _dptr(a))
        return r

    def name(self):
        return type(self).__name__

    def young_rows(self):
        """Young rows of the irrep (the probe for traced loops)."""
        raise NotImplementedError


class FundamentalRep(Representation):
    """D(U) = U, d = N (src/rep/rep_fundamental.hpp:15-25)."""
    kind = _lib.REP_FUND

    def __init__(self, N):
        super().__init__(N, N)

    def young_rows(self):
        return [1]

    def name(self):
        return "fundamental"


class AdjointRep(Representation):
    """Real orthogonal D_ab = 2 Tr(T^a U T^b U^dag), d = N^2-1 (src/rep/rep_adjoint.hpp:10-41)."""
    kind = _lib.REP_ADJ
    real = True

    def __init__(self, N):
        super().__init__(N, N * N - 1)

    def young_rows(self):
        return [2] + [1] * (self.N - 2)

    def name(self):
        return "adjoint"


class GeneralRep(Representation):
    """Irrep from Young rows (src/rep/rep_general.hpp:54-84); tables built by the library
    (gh_rep_general_build) or supplied, e.g. from the reference's own GeneralRep."""
    kind = _lib.REP_GENERAL

    def __init__(self, N, rows, real=False, T=None, W=None):
        rows = [int(r) for r in rows]
        rr = (C.c_int * len(rows))(*rows)
        d, n = C.c_int(), C.c_int()
        dimT = C.c_long()
        check(LIB.gh_rep_general_info(N, rr, len(rows), C.byref(d), C.byref(n), C.byref(dimT)))
        super().__init__(N, d.value)
        self.rows, self.real, self.n_boxes, self.dimT = rows, bool(real), n.value, dimT.value
        if T is None or W is None:
            T = np.zeros((N * N - 1, self.d, self.d), np.complex128)
            W = np.zeros((self.d, self.dimT), np.complex128)
            check(LIB.gh_rep_general_build(N, rr, len(rows), _dptr(T.view(np.float64)), _dptr(W.view(np.float64))))
        self.T = np.ascontiguousarray(T, np.complex128)
        self.W = np.ascontiguousarray(W, np.complex128)
        self.nality = self.n_boxes % N

    @classmethod
    def from_spec(cls, N, spec):
        """The reference driver's spec syntax "r1,r2[:real]" (src/hmc_higgs.cpp:21-34)."""
        real = False
        if ":" in spec:
            spec, tail = spec.split(":", 1)
            real = tail == "real"
        return cls(N, [int(t) for t in spec.split(",") if t], real)

    def young_rows(self):
        return list(self.rows)

    def closed_form_matrix(self, U):
        """D(U) of a single-row irrep in closed form (host; gh_sympow_matrix), with the
        number of monomial terms; raises GaugeHiggsError for irreps without one."""
        U = np.ascontiguousarray(U, np.complex128)
        Dm = np.zeros((self.d, self.d), np.complex128)
        nt = C.c_long()
        r = self.desc()
        check(LIB.gh_sympow_matrix(self.N, C.byref(r), _dptr(U.view(np.float64)), _dptr(Dm.view(np.float64)),
                                   C.byref(nt)))
        return Dm, nt.value

    def product_matrix(self, U):
        """D(U) as Q^dag (D_adj(U) (x)...) Q for irreps inside the adjoint's one- or
        two-fold product (host; gh_rep_product_matrix), with the number of adjoint
        factors K; raises GaugeHiggsError for irreps outside it."""
        U = np.ascontiguousarray(U, np.complex128)
        Dm = np.zeros((self.d, self.d), np.complex128)
        K = C.c_int()
        r = self.desc()
        check(LIB.gh_rep_product_matrix(self.N, C.byref(r), _dptr(U.view(np.float64)), _dptr(Dm.view(np.float64)),
                                        C.byref(K)))
        return Dm, K.value

    def name(self):
        return "general[" + ",".join(map(str, self.rows)) + "]"


def make_rep(N, spec):
    """src/hmc_higgs.cpp:23-34: "fund" | "adj" | Young rows with optional ":real"."""
    if spec == "fund":
        return FundamentalRep(N)
    if spec == "adj":
        return AdjointRep(N)
    return GeneralRep.from_spec(N, spec)


# ---------------------------------------------------------------------------
# Multi-invariant onsite potential (src/action/scalar_invariants.hpp)
# ---------------------------------------------------------------------------
class CasimirChannels:
    """The quartic channels of R (x) Rbar: distinct eigenvalues C2 of the adjoint Casimir
    superoperator sum_a [T^a_R, [T^a_R, .]], ascending (CasimirChannels<N>,
    src/action/scalar_invariants.hpp:19-27).  Couplings f_c are given in this order."""

    def __init__(self, rep):
        self.rep = rep
        c2 = np.zeros(rep.d * rep.d + 1)
        n = C.c_int()
        check(LIB.gh_casimir_channels(rep.N, C.byref(rep.desc()), _dptr(c2), len(c2), C.byref(n)))
        self.c2 = c2[:n.value].copy()

    @property
    def lambda_(self):
        return self.c2

    def n_channels(self):
        return len(self.c2)

    def superop(self, f):
        """A = sum_c 2 f_c P_c as a (d^2, d^2) complex matrix, vec index i*d + j."""
        f = np.ascontiguousarray(f, np.float64)
        d = self.rep.d
        A = np.zeros((d * d, d * d), np.complex128)
        check(LIB.gh_multi_superop(self.rep.N, C.byref(self.rep.desc()), len(f), _dptr(f), _dptr(A.view(np.float64))))
        return A


class MultiInvariantPotential:
    """V = -mu2 phi^dag phi + sum_c f_c Tr(M^dag P_c M), M = phi phi^dag
    (MultiInvariantPotential<N>, src/action/scalar_invariants.hpp:190-206).  Plug it in
    with `hmc.potential = pot`; `hmc.potential = None` restores the quartic potential."""

    def __init__(self, channels, f, mu2):
        self.ch = channels
        self.f = np.ascontiguousarray(f, np.float64)
        self.mu2 = float(mu2)
        if len(self.f) != channels.n_channels():
            raise ValueError(f"need {channels.n_channels()} couplings, got {len(self.f)}")

    def superop(self):
        return self.ch.superop(self.f)

    def value(self, phi):
        """V of one d-vector (host evaluation through the same superoperator)."""
        phi = np.asarray(phi, np.complex128)
        w = (self.superop() @ np.outer(phi, phi.conj()).reshape(-1)).reshape(len(phi), len(phi)) @ phi
        return -self.mu2 * float(np.vdot(phi, phi).real) + 0.5 * float(np.vdot(phi, w).real)


# ---------------------------------------------------------------------------
# Engine context
# ---------------------------------------------------------------------------
class _Context:
    def __init__(self, D, N, extents, rep, seeds, precision):
        n_lat = len(extents)
        L = (C.c_int * (n_lat * D))(*[int(x) for e in extents for x in e])
        sd = (C.c_uint64 * n_lat)(*[int(s) for s in seeds])
        self._rep_desc = rep.desc() if rep is not None else None
        out = C.c_void_p()
        check(LIB.gh_ctx_create(D, N, n_lat, L, C.byref(self._rep_desc) if rep is not None else None,
                                _PREC[precision], sd, C.byref(out)))
        self.h = out

    def close(self):
        if self.h:
            LIB.gh_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __call__(self, fn, *args):
        return check(getattr(LIB, fn)(self.h, *args), self.h)


class Ensemble:
    """n_lat independent lattices (equal D, N and representation; extents, couplings and
    seeds per lattice) evolved together: every kernel launch covers all lattices, each
    trajectory of the whole ensemble is one CUDA graph launch."""

    def __init__(self, extents, rep=None, seeds=None, D=None, N=None, precision="fp64",
                 beta=2.3, kappa=0.1, lam=0.5, tau=1.0, nmd=20, integ="omelyan"):
        extents = [list(e) for e in extents]
        self.D = D or len(extents[0])
        self.N = N or (rep.N if rep is not None else 3)
        if rep is not None and rep.N != self.N:
            raise ValueError("representation N differs from the gauge group N")
        self.rep = rep
        self.extents = extents
        self.n_lat = len(extents)
        seeds = seeds if seeds is not None else [1] * self.n_lat
        self.precision = precision
        self.ctx = _Context(self.D, self.N, extents, rep, seeds, precision)
        self.V = [int(np.prod(e)) for e in extents]
        self.d = rep.d if rep is not None else 0
        self._tau, self._nmd, self._integ = tau, nmd, _INTEG[integ]
        self.ctx("gh_set_integrator", self._integ, self._nmd, self._tau)
        b = np.broadcast_to(np.asarray(beta, float), (self.n_lat,))
        k = np.broadcast_to(np.asarray(kappa, float), (self.n_lat,))
        lm = np.broadcast_to(np.asarray(lam, float), (self.n_lat,))
        for i in range(self.n_lat):
            self.ctx("gh_set_couplings", i, float(b[i]), float(k[i]), float(lm[i]))

    # ---- onsite potential ----
    @property
    def potential(self):
        return getattr(self, "_potential", None)

    @potential.setter
    def potential(self, pot):
        """GaugeHiggsHMC::potential (src/hmc/gauge_higgs_hmc.hpp:25-27): a
        MultiInvariantPotential for every lattice, or None for the quartic potential."""
        if pot is None:
            self.ctx("gh_set_potential_quartic")
        else:
            self.ctx("gh_set_potential_multi", len(pot.f), _dptr(pot.f), pot.mu2)
        self._potential = pot

    # ---- loops traced in a probe irrep (src/measure/observables.hpp:36-101) ----
    def _rows(self, rep):
        if rep is None:
            return None, 0
        rows = rep.young_rows() if hasattr(rep, "young_rows") else list(rep)
        return (C.c_int * len(rows))(*rows), len(rows)

    def wilson_loop(self, Ra, Rb, rep=None, lat=-1):
        """<(1/d_R) Re Tr D^R(W_loop)> of the Ra x Rb rectangles (wilson_loop_fund when rep is
        None, wilson_loop_rep otherwise); rep: a Representation or Young rows."""
        rows, m = self._rows(rep)
        out = np.zeros(self.n_lat if lat < 0 else 1)
        self.ctx("gh_wilson_loop", lat, int(Ra), int(Rb), rows, m, _dptr(out))
        return out if lat < 0 and self.n_lat > 1 else float(out[0])

    def polyakov_loop_rep(self, rep=None, tdir=-1, lat=-1):
        """<(1/d_R) Re Tr D^R(prod_t U_tdir)> (polyakov_loop_rep)."""
        rows, m = self._rows(rep)
        out = np.zeros(self.n_lat if lat < 0 else 1)
        self.ctx("gh_polyakov_rep", lat, int(tdir), rows, m, _dptr(out))
        return out if lat < 0 and self.n_lat > 1 else float(out[0])

    # ---- frozen-length scalar ----
    @property
    def frozen_phi(self):
        return getattr(self, "_frozen", False)

    @frozen_phi.setter
    def frozen_phi(self, on):
        """GaugeHiggsHMC::frozen_phi (src/hmc/gauge_higgs_hmc.hpp:38-40): |phi_x| = 1
        HMC with tangent-space momenta and the great-circle scalar drift."""
        self.ctx("gh_set_frozen_phi", 1 if on else 0)
        self._frozen = bool(on)

    def normalize_phi(self):
        """Put every site on the unit sphere (src/hmc/gauge_higgs_hmc.hpp:73-82)."""
        self.ctx("gh_normalize_phi")

    # ---- couplings / integrator ----
    def set_couplings(self, lat, beta, kappa, lam):
        self.ctx("gh_set_couplings", lat, beta, kappa, lam)

    def couplings(self, lat):
        b, k, l = C.c_double(), C.c_double(), C.c_double()
        self.ctx("gh_get_couplings", lat, C.byref(b), C.byref(k), C.byref(l))
        return b.value, k.value, l.value

    def set_integrator(self, integ=None, nmd=None, tau=None):
        if integ is not None:
            self._integ = _INTEG[integ]
        if nmd is not None:
            self._nmd = int(nmd)
        if tau is not None:
            self._tau = float(tau)
        self.ctx("gh_set_integrator", self._integ, self._nmd, self._tau)

    def traj_counts(self, lat):
        t, a, nf = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.ctx("gh_get_traj_count", lat, C.byref(t), C.byref(a), C.byref(nf))
        return t.value, a.value, nf.value

    def set_traj_count(self, lat, traj, accepted=0):
        self.ctx("gh_set_traj_count", lat, int(traj), int(accepted))

    # ---- fields ----
    def _shape(self, kind, lat):
        V = self.V[lat]
        return {"U": (V, self.D, self.N, self.N), "P": (V, self.D, self.N * self.N - 1),
                "phi": (V, self.d), "pi": (V, self.d)}[kind]

    def get(self, kind, lat=0):
        shape = self._shape(kind, lat)
        if kind == "P":
            out = np.zeros(shape, np.float64)
            self.ctx("gh_get_mom", lat, _dptr(out))
            return out
        out = np.zeros(shape, np.complex128)
        fn = {"U": "gh_get_links", "phi": "gh_get_phi", "pi": "gh_get_pi"}[kind]
        self.ctx(fn, lat, _dptr(out.view(np.float64)))
        return out

    def set(self, kind, value, lat=0):
        shape = self._shape(kind, lat)
        if kind == "P":
            a = np.ascontiguousarray(np.broadcast_to(value, shape), np.float64)
            self.ctx("gh_set_mom", lat, _dptr(a))
            return
        a = np.ascontiguousarray(np.broadcast_to(value, shape), np.complex128)
        fn = {"U": "gh_set_links", "phi": "gh_set_phi", "pi": "gh_set_pi"}[kind]
        self.ctx(fn, lat, _dptr(a.view(np.float64)))

    # ---- initialisation (counter RNG, per-lattice seeds) ----
    def hot(self, sigma=1.0):
        self.ctx("gh_hot_start", float(sigma))

    def cold(self):
        self.ctx("gh_cold_start")

    def phi_gaussian(self, stream, sigma=1.0):
        self.ctx("gh_phi_gaussian", int(stream), float(sigma))

    def phi_cold(self, c=1.0):
        self.ctx("gh_phi_cold", float(c))

    def mom_refresh(self, stream):
        self.ctx("gh_mom_refresh", int(stream))

    def refresh_momenta(self):
        self.ctx("gh_refresh_momenta")

    # ---- MD ----
    def kick(self, eps):
        self.ctx("gh_kick", float(eps))

    def drift(self, eps):
        self.ctx("gh_drift", float(eps))

    def md_evolve(self):
        self.ctx("gh_md_evolve")

    def reunitarize_all(self):
        self.ctx("gh_reunitarize")

    def sync(self):
        self.ctx("gh_sync")

    # ---- forces (one lattice) ----
    def gauge_force(self, lat=0):
        F = np.zeros(self._shape("P", lat))
        self.ctx("gh_gauge_force", lat, _dptr(F))
        return F

    def matter_link_force(self, lat=0):
        F = np.zeros(self._shape("P", lat))
        self.ctx("gh_matter_link_force", lat, _dptr(F))
        return F

    def scalar_force(self, lat=0):
        F = np.zeros(self._shape("phi", lat), np.complex128)
        self.ctx("gh_scalar_force", lat, _dptr(F.view(np.float64)))
        return F

    # ---- measurements ----
    def measure(self, lat=0):
        o = Obs()
        self.ctx("gh_measure", lat, C.byref(o))
        return {k: getattr(o, k) for k, _ in Obs._fields_}

    def measure_all(self):
        arr = (Obs * self.n_lat)()
        self.ctx("gh_measure", -1, arr)
        return [{k: getattr(o, k) for k, _ in Obs._fields_} for o in arr]

    def polyakov_loop(self, lat=0, tdir=None):
        out = C.c_double()
        self.ctx("gh_polyakov", lat, self.D - 1 if tdir is None else tdir, C.byref(out))
        return out.value

    # ---- trajectories ----
    def trajectory(self):
        dH = np.zeros(self.n_lat)
        acc = np.zeros(self.n_lat, np.int32)
        self.ctx("gh_trajectory", _dptr(dH), acc.ctypes.data_as(C.POINTER(C.c_int)))
        return dH, acc.astype(bool)

    def run(self, ntraj, records=True):
        """ntraj trajectories back to back; returns a structured array [ntraj, n_lat]."""
        if not records:
            self.ctx("gh_run_trajectories", int(ntraj), None)
            return None
        recs = (TrajRecord * (ntraj * self.n_lat))()
        self.ctx("gh_run_trajectories", int(ntraj), recs)
        dt = np.dtype(TRAJ_DTYPE)
        arr = np.frombuffer(recs, dtype=dt, count=ntraj * self.n_lat).copy()
        return arr.reshape(ntraj, self.n_lat)

    def enqueue(self, ntraj=1):
        """Enqueue trajectories on the context stream without synchronising."""
        self.ctx("gh_enqueue_trajectories", int(ntraj))

    def records(self, ntraj):
        """Records of the last ntraj (<= 1024) trajectories, [ntraj, n_lat]."""
        recs = (TrajRecord * (ntraj * self.n_lat))()
        self.ctx("gh_read_records", int(ntraj), recs)
        dt = np.dtype(TRAJ_DTYPE)
        return np.frombuffer(recs, dtype=dt, count=ntraj * self.n_lat).copy().reshape(ntraj, self.n_lat)

    def autotune(self, reps=3):
        """Pick the kick tile of every group of equal-extent lattices by timing."""
        ms = C.c_double()
        self.ctx("gh_autotune", int(reps), C.byref(ms))
        return ms.value

    def set_tile(self, tile, lat=-1):
        t = (C.c_int * 4)(*(list(tile) + [1] * (4 - len(tile))))
        self.ctx("gh_set_tile", lat, t)

    def get_tile(self, lat=0):
        t = (C.c_int * 4)()
        self.ctx("gh_get_tile", lat, t)
        return list(t)[:self.D]

    def use_graph(self, on=True):
        self.ctx("gh_use_graph", int(bool(on)))

    # ---- tempering ----
    def enable_tempering(self, on=True, swap_seed=0x5A7AB1EC, coupling="kappa"):
        """Replica tempering across equal-extent lattices (src/hmc/replica_tempering.hpp):
        coupling "beta" (the reference's) or "kappa"."""
        mode = {"kappa": 1, "beta": 2}[coupling] if on else 0
        self.ctx("gh_temper_enable", mode, int(swap_seed))

    def set_temper_interval(self, n_sweep):
        """One swap pass after every n_sweep trajectories (ReplicaTempering::n_sweep)."""
        self.ctx("gh_temper_interval", int(n_sweep))

    def tempering_stats(self):
        att = np.zeros(max(self.n_lat - 1, 1), np.uint64)
        acc = np.zeros(max(self.n_lat - 1, 1), np.uint64)
        kap = np.zeros(self.n_lat)
        self.ctx("gh_temper_stats", att.ctypes.data_as(C.POINTER(C.c_uint64)),
                 acc.ctypes.data_as(C.POINTER(C.c_uint64)), _dptr(kap))
        return att, acc, kap

    _PATHS = {0: "register", 1: "tensor", 2: "closed_form", 3: "product", 4: "pair"}

    def rep_path(self):
        """How the device applies D(U): "register" (fundamental, adjoint), "tensor"
        (general irreps), "closed_form" (large single-row irreps), "product" (irreps
        inside the adjoint's one- or two-fold product, e.g. the SU(3) octet and 27-plet)
        or "pair" (two-slot irreps outside it, e.g. the SU(3) sextet and antitriplet)."""
        p = C.c_int()
        self.ctx("gh_rep_path", C.byref(p))
        return self._PATHS[p.value]

    def set_rep_path(self, path):
        """Switch a general irrep between "product" or "pair" and the path it takes without them."""
        code = {v: k for k, v in self._PATHS.items()}[path]
        self.ctx("gh_set_rep_path", code)

    def device_bytes(self):
        b = C.c_uint64()
        self.ctx("gh_device_bytes", C.byref(b))
        return b.value

    def set_stream(self, stream_ptr):
        self.ctx("gh_set_stream", C.c_void_p(stream_ptr))

    def close(self):
        self.ctx.close()


class GaugeHiggsHMC(Ensemble):
    """Single-lattice gauge + Higgs HMC (src/hmc/gauge_higgs_hmc.hpp:15-195)."""

    def __init__(self, extents, rep, seed=1, precision="fp64", beta=2.3, kappa=0.1, lam=0.5, tau=1.0, nmd=20,
                 integ="omelyan", D=None, N=None):
        super().__init__([extents], rep, [seed], D=D or len(extents), N=N or (rep.N if rep else None),
                         precision=precision, beta=beta, kappa=kappa, lam=lam, tau=tau, nmd=nmd, integ=integ)
        self.last_dH = 0.0

    # reference member names
    @property
    def U(self):
        return self.get("U")

    @U.setter
    def U(self, v):
        self.set("U", v)

    @property
    def P(self):
        return self.get("P")

    @P.setter
    def P(self, v):
        self.set("P", v)

    @property
    def phi(self):
        return self.get("phi")

    @phi.setter
    def phi(self, v):
        self.set("phi", v)

    @property
    def pi(self):
        return self.get("pi")

    @pi.setter
    def pi(self, v):
        self.set("pi", v)

    @property
    def beta(self):
        return self.couplings(0)[0]

    @beta.setter
    def beta(self, v):
        b, k, l = self.couplings(0)
        self.set_couplings(0, v, k, l)

    @property
    def kappa(self):
        return self.couplings(0)[1]

    @kappa.setter
    def kappa(self, v):
        b, k, l = self.couplings(0)
        self.set_couplings(0, b, v, l)

    @property
    def lam(self):
        return self.couplings(0)[2]

    @lam.setter
    def lam(self, v):
        b, k, l = self.couplings(0)
        self.set_couplings(0, b, k, v)

    @property
    def nmd(self):
        return self._nmd

    @nmd.setter
    def nmd(self, v):
        self.set_integrator(nmd=v)

    @property
    def tau(self):
        return self._tau

    @tau.setter
    def tau(self, v):
        self.set_integrator(tau=v)

    @property
    def integ(self):
        return self._integ

    @integ.setter
    def integ(self, v):
        self.set_integrator(integ=v)

    @property
    def traj_count(self):
        return self.traj_counts(0)[0]

    @traj_count.setter
    def traj_count(self, v):
        t, a, _ = self.traj_counts(0)
        self.set_traj_count(0, v, a)

    @property
    def accept_count(self):
        return self.traj_counts(0)[1]

    def reset_counters(self):
        """hmc.traj_count = 0; hmc.accept_count = 0 (src/hmc_higgs.cpp:76)."""
        self.set_traj_count(0, 0, 0)

    def acceptance(self):
        t, a, _ = self.traj_counts(0)
        return a / t if t else 0.0

    def hamiltonian(self):
        return self.measure(0)["H"]

    def gauge_action(self):
        return self.measure(0)["S_g"]

    def scalar_action(self):
        return self.measure(0)["S_H"]

    def avg_plaquette(self):
        return self.measure(0)["plaquette"]

    def link_energy(self):
        return self.measure(0)["L_link"]

    def higgs_length(self):
        return self.measure(0)["L_phi"]

    def trajectory(self):
        dH, acc = super().trajectory()
        self.last_dH = float(dH[0])
        return bool(acc[0])

    def trajectory_host(self, U, phi):
        """One trajectory on host-resident fields (updated in place); returns the record."""
        rec = TrajRecord()
        Uf = U.view(np.float64)
        pf = phi.view(np.float64) if phi is not None else None
        self.ctx("gh_trajectory_host", _dptr(Uf), _dptr(pf) if pf is not None else None, C.byref(rec))
        return rec


class GaugeHMC(GaugeHiggsHMC):
    """Pure-gauge HMC (src/hmc/hmc.hpp:12-96)."""

    def __init__(self, extents, N, seed=1, precision="fp64", beta=2.3, tau=1.0, nmd=20, integ="omelyan"):
        Ensemble.__init__(self, [extents], None, [seed], D=len(extents), N=N, precision=precision, beta=beta,
                          kappa=0.0, lam=0.0, tau=tau, nmd=nmd, integ=integ)
        self.last_dH = 0.0
