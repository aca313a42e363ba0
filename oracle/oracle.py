"""ctypes front end of the parity checker -- TEST INFRASTRUCTURE ONLY.

Two back ends share one calling convention (numpy arrays in the reference's
array-of-structures layouts, complex as interleaved float64 pairs):

* ``Oracle`` -- oracle/_build/libghoracle.so, the plain-C restatement
  (oracle/gh_oracle.c).  Always available once oracle/Makefile has run.
* ``Reference`` -- oracle/_ref/libghref.so, the unmodified reference headers
  behind oracle/ref_harness.cpp.  Present where it was built (it is built from
  the reference sources, which exist only in the development container; the
  built library travels with the repository snapshot).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The product (gauge_higgs_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libghoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libghref.so")
REF_NOFMA_SO = os.path.join(HERE, "_ref", "libghref_nofma.so")

REP_NONE, REP_FUND, REP_ADJ, REP_GENERAL = 0, 1, 2, 3
LEAPFROG, OMELYAN = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u64 = C.c_uint64


def _d(a):
    return a.ctypes.data_as(_dp)


def _cplx(a):
    """complex128 array -> contiguous float64 view (interleaved re, im)."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.view(np.float64)


def ng(N):
    return N * N - 1


# --------------------------------------------------------------------------
# C restatement
# --------------------------------------------------------------------------
class _Lattice(C.Structure):
    _fields_ = [("D", C.c_int), ("N", C.c_int), ("L", C.c_int * 4), ("vol", C.c_int64),
                ("stride", C.c_int64 * 4)]


class _Rep(C.Structure):
    _fields_ = [("kind", C.c_int), ("N", C.c_int), ("d", C.c_int), ("real", C.c_int),
                ("n", C.c_int), ("dimT", C.c_long), ("T", _dp), ("W", _dp)]


class _Hmc(C.Structure):
    _fields_ = [("lat", _Lattice), ("rep", C.POINTER(_Rep)), ("seed", _u64),
                ("beta", C.c_double), ("kappa", C.c_double), ("lambda_", C.c_double), ("tau", C.c_double),
                ("nmd", C.c_int), ("integ", C.c_int), ("reunit_each_traj", C.c_int),
                ("traj_count", _u64), ("accept_count", _u64), ("last_dH", C.c_double),
                ("U", _dp), ("P", _dp), ("phi", _dp), ("pi", _dp)]


class OracleRep:
    """A representation for the oracle: kind + (for general irreps) T_R and W tables."""

    def __init__(self, lib, kind, N, d=0, real=0, n=0, dimT=0, T=None, W=None):
        self._lib = lib
        self.s = _Rep()
        self._T = None if T is None else _cplx(T)
        self._W = None if W is None else _cplx(W)
        lib.gho_rep_init(C.byref(self.s), kind, N, d, real, n, dimT,
                         _d(self._T) if self._T is not None else None,
                         _d(self._W) if self._W is not None else None)
        self.kind, self.N, self.d, self.real = kind, N, self.s.d, self.s.real

    def __del__(self):
        try:
            self._lib.gho_rep_free(C.byref(self.s))
        except Exception:
            pass


class Oracle:
    """FP64 single-thread C restatement of the reference MD path."""

    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        L.gho_splitmix64.restype = _u64
        L.gho_splitmix64.argtypes = [_u64]
        L.gho_key.restype = _u64
        L.gho_key.argtypes = [_u64] * 5
        L.gho_uniform.restype = C.c_double
        L.gho_uniform.argtypes = [_u64, _u64]
        L.gho_gauss.restype = C.c_double
        L.gho_gauss.argtypes = [_u64, _u64]
        for f in ("gho_gauge_action", "gho_scalar_action"):
            getattr(L, f).restype = C.c_double
        L.gho_gauge_action.argtypes = [C.c_void_p, _dp, C.c_double]
        L.gho_avg_plaquette.restype = C.c_double
        L.gho_avg_plaquette.argtypes = [C.c_void_p, _dp]
        L.gho_add_gauge_force.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
        L.gho_scalar_action.argtypes = [C.c_void_p, C.c_void_p, _dp, _dp, C.c_double, C.c_double]
        L.gho_scalar_force.argtypes = [C.c_void_p, C.c_void_p, _dp, _dp, C.c_double, C.c_double, _dp]
        L.gho_add_matter_link_force.argtypes = [C.c_void_p, C.c_void_p, _dp, _dp, C.c_double, _dp]
        L.gho_link_energy.restype = C.c_double
        L.gho_scalar_action_multi.restype = C.c_double
        L.gho_scalar_action_multi.argtypes = [C.c_void_p, C.c_void_p, _dp, _dp, C.c_double, _dp, C.c_double]
        L.gho_scalar_force_multi.argtypes = [C.c_void_p, C.c_void_p, _dp, _dp, C.c_double, _dp, C.c_double, _dp]
        L.gho_multi_potential.argtypes = [C.c_int, _dp, C.c_double, _dp, _dp, _dp]
        L.gho_link_energy.argtypes = [C.c_void_p, C.c_void_p, _dp, _dp]
        L.gho_higgs_length.restype = C.c_double
        L.gho_higgs_length.argtypes = [C.c_void_p, C.c_int, _dp]
        L.gho_polyakov.restype = C.c_double
        L.gho_polyakov.argtypes = [C.c_void_p, _dp, C.c_int]
        L.gho_kinetic_mom.restype = C.c_double
        L.gho_kinetic_mom.argtypes = [C.c_void_p, _dp]
        L.gho_kinetic_vec.restype = C.c_double
        L.gho_kinetic_vec.argtypes = [C.c_void_p, C.c_int, _dp]
        L.gho_hot_start.argtypes = [C.c_void_p, _u64, C.c_double, _dp]
        L.gho_phi_gaussian.argtypes = [C.c_void_p, C.c_int, _u64, _u64, C.c_int, C.c_double, _dp]
        L.gho_mom_refresh.argtypes = [C.c_void_p, _u64, _u64, _dp]
        L.gho_rep_init.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_long, _dp, _dp]
        L.gho_rep_rotate.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int]
        L.gho_rep_hop_link_g.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.gho_rep_matrix.argtypes = [C.c_void_p, _dp, _dp]
        L.gho_expi.argtypes = [C.c_int, _dp, _dp]
        L.gho_reunitarize.argtypes = [C.c_int, _dp]
        L.gho_generators.argtypes = [C.c_int, _dp]
        L.gho_structure_constants.argtypes = [C.c_int, _dp]
        L.gho_hmc_init.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, C.c_void_p, _u64]
        L.gho_hmc_hamiltonian.restype = C.c_double
        L.gho_hmc_hamiltonian.argtypes = [C.c_void_p]
        L.gho_hmc_kick.argtypes = [C.c_void_p, C.c_double]
        L.gho_hmc_drift.argtypes = [C.c_void_p, C.c_double]
        for f in ("gho_hmc_md_evolve", "gho_hmc_refresh_momenta", "gho_hmc_reunitarize_all", "gho_hmc_free"):
            getattr(L, f).argtypes = [C.c_void_p]
        L.gho_hmc_trajectory.restype = C.c_int
        L.gho_hmc_trajectory.argtypes = [C.c_void_p]

    # ---- helpers ----
    def lattice(self, D, N, L):
        lat = _Lattice()
        arr = (C.c_int * 4)(*list(L) + [1] * (4 - len(L)))
        self.lib.gho_lattice_init(C.byref(lat), D, N, arr)
        return lat

    def rep(self, kind, N, d=0, real=0, n=0, dimT=0, T=None, W=None):
        return OracleRep(self.lib, kind, N, d, real, n, dimT, T, W)

    # ---- RNG ----
    def key(self, a, b=0, c=0, d=0, e=0):
        return self.lib.gho_key(a, b, c, d, e)

    def uniform(self, seed, k):
        return self.lib.gho_uniform(seed, k)

    def gauss(self, seed, k):
        return self.lib.gho_gauss(seed, k)

    # ---- group ----
    def generators(self, N):
        T = np.zeros((ng(N), N, N), np.complex128)
        self.lib.gho_generators(N, _d(T.view(np.float64)))
        return T

    def structure_constants(self, N):
        f = np.zeros((ng(N),) * 3)
        self.lib.gho_structure_constants(N, _d(f))
        return f

    def expi(self, H):
        H = np.ascontiguousarray(H, np.complex128)
        U = np.zeros_like(H)
        self.lib.gho_expi(H.shape[0], _d(H.view(np.float64)), _d(U.view(np.float64)))
        return U

    def reunitarize(self, U):
        U = np.array(U, np.complex128, copy=True)
        self.lib.gho_reunitarize(U.shape[0], _d(U.view(np.float64)))
        return U

    # ---- fields (shapes: U [V,D,N,N] c128, P [V,D,ng] f64, phi [V,d] c128) ----
    def hot_start(self, D, N, L, seed, sigma):
        lat = self.lattice(D, N, L)
        U = np.zeros((lat.vol, D, N, N), np.complex128)
        self.lib.gho_hot_start(C.byref(lat), seed, sigma, _d(U.view(np.float64)))
        return U

    def phi_gaussian(self, D, L, d, seed, stream, real, sigma):
        lat = self.lattice(D, 2, L)
        phi = np.zeros((lat.vol, d), np.complex128)
        self.lib.gho_phi_gaussian(C.byref(lat), d, seed, stream, int(real), sigma, _d(phi.view(np.float64)))
        return phi

    def mom_refresh(self, D, N, L, seed, stream):
        lat = self.lattice(D, N, L)
        P = np.zeros((lat.vol, D, ng(N)))
        self.lib.gho_mom_refresh(C.byref(lat), seed, stream, _d(P))
        return P

    def gauge_action(self, D, N, L, U, beta):
        lat = self.lattice(D, N, L)
        return self.lib.gho_gauge_action(C.byref(lat), _d(_cplx(U)), beta)

    def avg_plaquette(self, D, N, L, U):
        lat = self.lattice(D, N, L)
        return self.lib.gho_avg_plaquette(C.byref(lat), _d(_cplx(U)))

    def gauge_force(self, D, N, L, U, beta):
        lat = self.lattice(D, N, L)
        F = np.zeros((lat.vol, D, ng(N)))
        self.lib.gho_add_gauge_force(C.byref(lat), _d(_cplx(U)), beta, _d(F))
        return F

    def matter_force(self, D, N, L, rep, U, phi, kappa):
        lat = self.lattice(D, N, L)
        F = np.zeros((lat.vol, D, ng(N)))
        self.lib.gho_add_matter_link_force(C.byref(lat), C.byref(rep.s), _d(_cplx(U)), _d(_cplx(phi)), kappa, _d(F))
        return F

    def scalar_force(self, D, N, L, rep, U, phi, kappa, lam):
        lat = self.lattice(D, N, L)
        Fp = np.zeros((lat.vol, rep.d), np.complex128)
        self.lib.gho_scalar_force(C.byref(lat), C.byref(rep.s), _d(_cplx(U)), _d(_cplx(phi)), kappa, lam,
                                  _d(Fp.view(np.float64)))
        return Fp

    def scalar_action(self, D, N, L, rep, U, phi, kappa, lam):
        lat = self.lattice(D, N, L)
        return self.lib.gho_scalar_action(C.byref(lat), C.byref(rep.s), _d(_cplx(U)), _d(_cplx(phi)), kappa, lam)

    def multi_potential(self, d, A, mu2, phi):
        A = np.ascontiguousarray(A, np.complex128)
        phi = np.ascontiguousarray(phi, np.complex128)
        g = np.zeros_like(phi)
        v = C.c_double()
        self.lib.gho_multi_potential(d, _d(A.view(np.float64)), mu2, _d(phi.view(np.float64)), C.byref(v),
                                     _d(g.view(np.float64)))
        return v.value, g

    def scalar_force_multi(self, D, N, L, rep, U, phi, kappa, A, mu2):
        lat = self.lattice(D, N, L)
        A = np.ascontiguousarray(A, np.complex128)
        Fp = np.zeros((lat.vol, rep.d), np.complex128)
        self.lib.gho_scalar_force_multi(C.byref(lat), C.byref(rep.s), _d(_cplx(U)), _d(_cplx(phi)), kappa,
                                        _d(A.view(np.float64)), mu2, _d(Fp.view(np.float64)))
        return Fp

    def scalar_action_multi(self, D, N, L, rep, U, phi, kappa, A, mu2):
        lat = self.lattice(D, N, L)
        A = np.ascontiguousarray(A, np.complex128)
        return self.lib.gho_scalar_action_multi(C.byref(lat), C.byref(rep.s), _d(_cplx(U)), _d(_cplx(phi)), kappa,
                                                _d(A.view(np.float64)), mu2)

    def link_energy(self, D, N, L, rep, U, phi):
        lat = self.lattice(D, N, L)
        return self.lib.gho_link_energy(C.byref(lat), C.byref(rep.s), _d(_cplx(U)), _d(_cplx(phi)))

    def higgs_length(self, D, L, phi):
        lat = self.lattice(D, 2, L)
        phi = np.ascontiguousarray(phi, np.complex128)
        return self.lib.gho_higgs_length(C.byref(lat), phi.shape[-1], _d(phi.view(np.float64)))

    def polyakov(self, D, N, L, U, tdir=None):
        lat = self.lattice(D, N, L)
        return self.lib.gho_polyakov(C.byref(lat), _d(_cplx(U)), D - 1 if tdir is None else tdir)

    def rep_rotate(self, rep, U, phi, dag=False):
        out = np.zeros(rep.d, np.complex128)
        self.lib.gho_rep_rotate(C.byref(rep.s), _d(_cplx(U)), _d(_cplx(phi)), _d(out.view(np.float64)), int(dag))
        return out

    def rep_hop(self, rep, U, phix, phiy):
        g = np.zeros(ng(rep.N))
        self.lib.gho_rep_hop_link_g(C.byref(rep.s), _d(_cplx(U)), _d(_cplx(phix)), _d(_cplx(phiy)), _d(g))
        return g

    def rep_matrix(self, rep, U):
        Dm = np.zeros((rep.d, rep.d), np.complex128)
        self.lib.gho_rep_matrix(C.byref(rep.s), _d(_cplx(U)), _d(Dm.view(np.float64)))
        return Dm

    def hmc(self, D, N, L, rep=None, seed=1, **kw):
        return OracleHMC(self, D, N, L, rep, seed, **kw)


class OracleHMC:
    """Oracle mirror of GaugeHiggsHMC / GaugeHMC (rep None -> pure gauge)."""

    def __init__(self, orc, D, N, L, rep, seed, beta=2.3, kappa=0.1, lam=0.5, tau=1.0, nmd=20,
                 integ=OMELYAN):
        self.o, self.D, self.N, self.L = orc, D, N, list(L)
        self.rep = rep
        self.h = _Hmc()
        Ls = (C.c_int * 4)(*list(L) + [1] * (4 - len(L)))
        orc.lib.gho_hmc_init(C.byref(self.h), D, N, Ls, C.byref(rep.s) if rep is not None else None, seed)
        self.V = int(self.h.lat.vol)
        self.d = rep.d if rep is not None else 1
        self.h.beta, self.h.kappa, self.h.lambda_, self.h.tau, self.h.nmd, self.h.integ = beta, kappa, lam, tau, nmd, integ

    def __del__(self):
        try:
            self.o.lib.gho_hmc_free(C.byref(self.h))
        except Exception:
            pass

    def _view(self, ptr, n):
        return np.ctypeslib.as_array(ptr, shape=(n,))

    @property
    def U(self):
        return self._view(self.h.U, self.V * self.D * self.N * self.N * 2).view(np.complex128).reshape(
            self.V, self.D, self.N, self.N)

    @property
    def P(self):
        return self._view(self.h.P, self.V * self.D * ng(self.N)).reshape(self.V, self.D, ng(self.N))

    @property
    def phi(self):
        return self._view(self.h.phi, self.V * self.d * 2).view(np.complex128).reshape(self.V, self.d)

    @property
    def pi(self):
        return self._view(self.h.pi, self.V * self.d * 2).view(np.complex128).reshape(self.V, self.d)

    def hamiltonian(self):
        return self.o.lib.gho_hmc_hamiltonian(C.byref(self.h))

    def kick(self, eps):
        self.o.lib.gho_hmc_kick(C.byref(self.h), eps)

    def drift(self, eps):
        self.o.lib.gho_hmc_drift(C.byref(self.h), eps)

    def md_evolve(self):
        self.o.lib.gho_hmc_md_evolve(C.byref(self.h))

    def refresh_momenta(self):
        self.o.lib.gho_hmc_refresh_momenta(C.byref(self.h))

    def reunitarize_all(self):
        self.o.lib.gho_hmc_reunitarize_all(C.byref(self.h))

    def trajectory(self):
        return bool(self.o.lib.gho_hmc_trajectory(C.byref(self.h)))


# --------------------------------------------------------------------------
# Reference harness
# --------------------------------------------------------------------------
class Reference:
    """The unmodified reference, driven through oracle/ref_harness.cpp."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: built by `make -C oracle ref` where the reference tree exists")
        L = self.lib = C.CDLL(path)
        L.ref_key.restype = _u64
        L.ref_key.argtypes = [_u64] * 5
        L.ref_uniform.restype = C.c_double
        L.ref_uniform.argtypes = [_u64, _u64]
        L.ref_gauss.restype = C.c_double
        L.ref_gauss.argtypes = [_u64, _u64]
        L.ref_gauss_many.argtypes = [_u64, C.POINTER(_u64), C.c_int64, _dp]
        L.ref_uniform_many.argtypes = [_u64, C.POINTER(_u64), C.c_int64, _dp]
        L.ref_rep_info.argtypes = [C.c_int, C.c_char_p, _ip, _ip, _ip, C.POINTER(C.c_long), _ip]
        L.ref_rep_tables.argtypes = [C.c_int, C.c_char_p, _dp, _dp]
        L.ref_rep_matrix.argtypes = [C.c_int, C.c_char_p, _dp, _dp]
        L.ref_rep_rotate.argtypes = [C.c_int, C.c_char_p, _dp, _dp, _dp, C.c_int]
        L.ref_rep_hop.argtypes = [C.c_int, C.c_char_p, _dp, _dp, _dp, _dp]
        L.ref_expi.argtypes = [C.c_int, _dp, _dp]
        L.ref_reunitarize.argtypes = [C.c_int, _dp]
        L.ref_generators.argtypes = [C.c_int, _dp]
        L.ref_hot_start.argtypes = [C.c_int, C.c_int, _ip, _u64, C.c_double, _dp]
        L.ref_mom_refresh.argtypes = [C.c_int, C.c_int, _ip, _u64, _u64, _dp]
        L.ref_phi_gaussian.argtypes = [C.c_int, _ip, C.c_int, _u64, _u64, C.c_int, C.c_double, _dp]
        for f in ("ref_gauge_action",):
            getattr(L, f).restype = C.c_double
        L.ref_gauge_action.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_double]
        L.ref_avg_plaquette.restype = C.c_double
        L.ref_avg_plaquette.argtypes = [C.c_int, C.c_int, _ip, _dp]
        L.ref_polyakov.restype = C.c_double
        L.ref_polyakov.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_int]
        L.ref_gauge_force.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_double, _dp]
        L.ref_matter_force.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, _dp, _dp, C.c_double, _dp]
        L.ref_scalar_force.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, _dp, _dp, C.c_double, C.c_double, _dp]
        L.ref_scalar_action.restype = C.c_double
        L.ref_scalar_action.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, _dp, _dp, C.c_double, C.c_double]
        L.ref_casimir_channels.argtypes = [C.c_int, C.c_char_p, _dp, C.c_int]
        L.ref_wilson_loop.restype = C.c_double
        L.ref_wilson_loop.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, _dp, C.c_int, C.c_int]
        L.ref_polyakov_rep.restype = C.c_double
        L.ref_polyakov_rep.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, _dp, C.c_int]
        L.ref_hmc_op_frozen.argtypes = [C.c_int, C.c_int, C.c_int, _ip, C.c_char_p, _u64, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, _u64, _dp, _dp, _dp,
                                        _dp, _dp]
        L.ref_multi_superop.argtypes = [C.c_int, C.c_char_p, _dp, C.c_int, C.c_double, _dp]
        L.ref_multi_value_dV.argtypes = [C.c_int, C.c_char_p, _dp, C.c_int, C.c_double, _dp, _dp, _dp]
        L.ref_scalar_force_multi.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, _dp, _dp, C.c_double, _dp, C.c_int,
                                             C.c_double, _dp]
        L.ref_scalar_action_multi.restype = C.c_double
        L.ref_scalar_action_multi.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, _dp, _dp, C.c_double, _dp, C.c_int,
                                              C.c_double]
        L.ref_link_energy.restype = C.c_double
        L.ref_link_energy.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, _dp, _dp]
        L.ref_hmc_op.argtypes = [C.c_int, C.c_int, C.c_int, _ip, C.c_char_p, _u64, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, _u64,
                                 _dp, _dp, _dp, _dp, _dp]
        L.ref_run.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, C.c_double, C.c_double, C.c_double,
                              C.c_int, C.c_int, C.c_int, C.c_double, _u64, C.c_int, C.c_double, C.c_double,
                              _dp, _dp]
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_set_threads.restype = C.c_int
        L.ref_session_create.restype = C.c_void_p
        L.ref_session_create.argtypes = [C.c_int, C.c_int, _ip, C.c_char_p, C.c_double, C.c_double, C.c_double,
                                         C.c_int, C.c_double, _u64, C.c_int, C.c_double, C.c_double]
        L.ref_session_run.argtypes = [C.c_void_p, C.c_int, _dp]
        L.ref_session_set_multi.argtypes = [C.c_void_p, _dp, C.c_int, C.c_double]
        L.ref_session_set_frozen.argtypes = [C.c_void_p, C.c_int]
        L.ref_session_acceptance.restype = C.c_double
        L.ref_session_acceptance.argtypes = [C.c_void_p]
        L.ref_session_destroy.argtypes = [C.c_void_p]

    @staticmethod
    def _L(L):
        return (C.c_int * 4)(*list(L) + [1] * (4 - len(L)))

    def set_threads(self, n):
        return self.lib.ref_set_threads(n)

    def key(self, a, b=0, c=0, d=0, e=0):
        return self.lib.ref_key(a, b, c, d, e)

    def uniform(self, seed, k):
        return self.lib.ref_uniform(seed, k)

    def gauss(self, seed, k):
        return self.lib.ref_gauss(seed, k)

    def gauss_many(self, seed, keys):
        keys = np.ascontiguousarray(keys, np.uint64)
        out = np.zeros(len(keys))
        self.lib.ref_gauss_many(seed, keys.ctypes.data_as(C.POINTER(_u64)), len(keys), _d(out))
        return out

    def uniform_many(self, seed, keys):
        keys = np.ascontiguousarray(keys, np.uint64)
        out = np.zeros(len(keys))
        self.lib.ref_uniform_many(seed, keys.ctypes.data_as(C.POINTER(_u64)), len(keys), _d(out))
        return out

    def rep_info(self, N, spec):
        d, real, n, uf = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        dimT = C.c_long()
        rc = self.lib.ref_rep_info(N, spec.encode(), C.byref(d), C.byref(real), C.byref(n), C.byref(dimT), C.byref(uf))
        if rc:
            raise ValueError(f"bad rep spec {spec}")
        return dict(d=d.value, real=real.value, n=n.value, dimT=dimT.value, use_fast=uf.value)

    def rep_tables(self, N, spec):
        info = self.rep_info(N, spec)
        d, dimT = info["d"], info["dimT"]
        T = np.zeros((ng(N), d, d), np.complex128)
        W = np.zeros((d, max(dimT, 1)), np.complex128)
        self.lib.ref_rep_tables(N, spec.encode(), _d(T.view(np.float64)), _d(W.view(np.float64)))
        return T, (W if dimT else None), info

    def rep_matrix(self, N, spec, U):
        d = self.rep_info(N, spec)["d"]
        Dm = np.zeros((d, d), np.complex128)
        self.lib.ref_rep_matrix(N, spec.encode(), _d(_cplx(U)), _d(Dm.view(np.float64)))
        return Dm

    def rep_rotate(self, N, spec, U, phi, dag=False):
        d = self.rep_info(N, spec)["d"]
        out = np.zeros(d, np.complex128)
        self.lib.ref_rep_rotate(N, spec.encode(), _d(_cplx(U)), _d(_cplx(phi)), _d(out.view(np.float64)), int(dag))
        return out

    def rep_hop(self, N, spec, U, phix, phiy):
        g = np.zeros(ng(N))
        self.lib.ref_rep_hop(N, spec.encode(), _d(_cplx(U)), _d(_cplx(phix)), _d(_cplx(phiy)), _d(g))
        return g

    def expi(self, H):
        H = np.ascontiguousarray(H, np.complex128)
        U = np.zeros_like(H)
        self.lib.ref_expi(H.shape[0], _d(H.view(np.float64)), _d(U.view(np.float64)))
        return U

    def reunitarize(self, U):
        U = np.array(U, np.complex128, copy=True)
        self.lib.ref_reunitarize(U.shape[0], _d(U.view(np.float64)))
        return U

    def generators(self, N):
        T = np.zeros((ng(N), N, N), np.complex128)
        self.lib.ref_generators(N, _d(T.view(np.float64)))
        return T

    def hot_start(self, D, N, L, seed, sigma):
        V = int(np.prod(L))
        U = np.zeros((V, D, N, N), np.complex128)
        self.lib.ref_hot_start(D, N, self._L(L), seed, sigma, _d(U.view(np.float64)))
        return U

    def mom_refresh(self, D, N, L, seed, stream):
        V = int(np.prod(L))
        P = np.zeros((V, D, ng(N)))
        self.lib.ref_mom_refresh(D, N, self._L(L), seed, stream, _d(P))
        return P

    def phi_gaussian(self, D, L, d, seed, stream, real, sigma):
        V = int(np.prod(L))
        phi = np.zeros((V, d), np.complex128)
        self.lib.ref_phi_gaussian(D, self._L(L), d, seed, stream, int(real), sigma, _d(phi.view(np.float64)))
        return phi

    def gauge_action(self, D, N, L, U, beta):
        return self.lib.ref_gauge_action(D, N, self._L(L), _d(_cplx(U)), beta)

    def avg_plaquette(self, D, N, L, U):
        return self.lib.ref_avg_plaquette(D, N, self._L(L), _d(_cplx(U)))

    def polyakov(self, D, N, L, U, tdir=None):
        return self.lib.ref_polyakov(D, N, self._L(L), _d(_cplx(U)), D - 1 if tdir is None else tdir)

    def gauge_force(self, D, N, L, U, beta):
        V = int(np.prod(L))
        F = np.zeros((V, D, ng(N)))
        self.lib.ref_gauge_force(D, N, self._L(L), _d(_cplx(U)), beta, _d(F))
        return F

    def matter_force(self, D, N, L, spec, U, phi, kappa):
        V = int(np.prod(L))
        F = np.zeros((V, D, ng(N)))
        self.lib.ref_matter_force(D, N, self._L(L), spec.encode(), _d(_cplx(U)), _d(_cplx(phi)), kappa, _d(F))
        return F

    def scalar_force(self, D, N, L, spec, U, phi, kappa, lam):
        phi = np.ascontiguousarray(phi, np.complex128)
        Fp = np.zeros_like(phi)
        self.lib.ref_scalar_force(D, N, self._L(L), spec.encode(), _d(_cplx(U)), _d(_cplx(phi)), kappa, lam,
                                  _d(Fp.view(np.float64)))
        return Fp

    def scalar_action(self, D, N, L, spec, U, phi, kappa, lam):
        return self.lib.ref_scalar_action(D, N, self._L(L), spec.encode(), _d(_cplx(U)), _d(_cplx(phi)), kappa, lam)

    def wilson_loop(self, D, N, L, spec, U, Ra, Rb):
        """spec "fund0": wilson_loop_fund; otherwise wilson_loop_rep in that irrep."""
        return self.lib.ref_wilson_loop(D, N, self._L(L), spec.encode(), _d(_cplx(U)), Ra, Rb)

    def polyakov_rep(self, D, N, L, spec, U, tdir):
        return self.lib.ref_polyakov_rep(D, N, self._L(L), spec.encode(), _d(_cplx(U)), tdir)

    # multi-invariant onsite potential (src/action/scalar_invariants.hpp)
    def casimir_channels(self, N, spec):
        c2 = np.zeros(256)
        n = self.lib.ref_casimir_channels(N, spec.encode(), _d(c2), len(c2))
        if n < 0:
            raise RuntimeError(f"ref_casimir_channels rc={n}")
        return c2[:n].copy()

    def multi_superop(self, N, spec, f, mu2):
        d = self.rep_info(N, spec)["d"] if spec not in ("fund", "adj") else (N if spec == "fund" else N * N - 1)
        f = np.ascontiguousarray(f, np.float64)
        A = np.zeros((d * d, d * d), np.complex128)
        rc = self.lib.ref_multi_superop(N, spec.encode(), _d(f), len(f), mu2, _d(A.view(np.float64)))
        if rc:
            raise RuntimeError(f"ref_multi_superop rc={rc}")
        return A

    def multi_value_dV(self, N, spec, f, mu2, phi):
        f = np.ascontiguousarray(f, np.float64)
        phi = np.ascontiguousarray(phi, np.complex128)
        g = np.zeros_like(phi)
        v = C.c_double()
        rc = self.lib.ref_multi_value_dV(N, spec.encode(), _d(f), len(f), mu2, _d(phi.view(np.float64)), C.byref(v),
                                         _d(g.view(np.float64)))
        if rc:
            raise RuntimeError(f"ref_multi_value_dV rc={rc}")
        return v.value, g

    def scalar_force_multi(self, D, N, L, spec, U, phi, kappa, f, mu2):
        phi = np.ascontiguousarray(phi, np.complex128)
        f = np.ascontiguousarray(f, np.float64)
        Fp = np.zeros_like(phi)
        rc = self.lib.ref_scalar_force_multi(D, N, self._L(L), spec.encode(), _d(_cplx(U)), _d(_cplx(phi)), kappa,
                                             _d(f), len(f), mu2, _d(Fp.view(np.float64)))
        if rc:
            raise RuntimeError(f"ref_scalar_force_multi rc={rc}")
        return Fp

    def scalar_action_multi(self, D, N, L, spec, U, phi, kappa, f, mu2):
        f = np.ascontiguousarray(f, np.float64)
        return self.lib.ref_scalar_action_multi(D, N, self._L(L), spec.encode(), _d(_cplx(U)), _d(_cplx(phi)), kappa,
                                                _d(f), len(f), mu2)

    def link_energy(self, D, N, L, spec, U, phi):
        return self.lib.ref_link_energy(D, N, self._L(L), spec.encode(), _d(_cplx(U)), _d(_cplx(phi)))

    def hmc_op(self, op, D, N, L, spec, state, seed=1, beta=2.3, kappa=0.1, lam=0.5, tau=1.0, nmd=20,
               integ=OMELYAN, eps=0.0, traj_count=0):
        """op: kick drift md_evolve hamiltonian refresh trajectory reunitarize.
        state: dict with U, P, phi, pi numpy arrays (modified in place)."""
        ops = dict(kick=0, drift=1, md_evolve=2, hamiltonian=3, refresh=4, trajectory=5, reunitarize=6)
        out = np.zeros(4)
        st = {k: np.ascontiguousarray(v) for k, v in state.items()}
        U = st["U"].view(np.float64)
        P = st["P"]
        phi = st["phi"].view(np.float64)
        pi = st["pi"].view(np.float64)
        rc = self.lib.ref_hmc_op(ops[op], D, N, self._L(L), spec.encode(), seed, beta, kappa, lam, tau, nmd, integ,
                                 eps, traj_count, _d(U), _d(P), _d(phi), _d(pi), _d(out))
        if rc:
            raise RuntimeError(f"ref_hmc_op rc={rc}")
        state.update(st)
        return out

    def hmc_op_frozen(self, op, D, N, L, spec, state, seed=1, beta=2.3, kappa=0.1, lam=0.5, tau=1.0, nmd=20,
                      integ=OMELYAN, eps=0.0, traj_count=0):
        """As hmc_op with GaugeHiggsHMC::frozen_phi on; op also "normalize"."""
        ops = dict(kick=0, drift=1, md_evolve=2, hamiltonian=3, refresh=4, trajectory=5, normalize=7)
        out = np.zeros(4)
        st = {k: np.ascontiguousarray(v) for k, v in state.items()}
        rc = self.lib.ref_hmc_op_frozen(ops[op], D, N, self._L(L), spec.encode(), seed, beta, kappa, lam, tau, nmd,
                                        integ, eps, traj_count, _d(st["U"].view(np.float64)), _d(st["P"]),
                                        _d(st["phi"].view(np.float64)), _d(st["pi"].view(np.float64)), _d(out))
        if rc:
            raise RuntimeError(f"ref_hmc_op_frozen rc={rc}")
        state.update(st)
        return out

    def run(self, D, N, L, spec, beta, kappa, lam, ntherm, nmeas, nmd, tau, seed, integ=OMELYAN,
            hot_sigma=0.8, phi_sigma=0.3):
        series = np.zeros((max(nmeas, 1), 5))
        acc = C.c_double()
        rc = self.lib.ref_run(D, N, self._L(L), spec.encode(), beta, kappa, lam, ntherm, nmeas, nmd, tau, seed,
                              integ, hot_sigma, phi_sigma, _d(series), C.byref(acc))
        if rc:
            raise RuntimeError(f"ref_run rc={rc}")
        return series[:nmeas], acc.value


class RefSession:
    """A persistent reference GaugeHiggsHMC driven by its own trajectory() loop."""

    def __init__(self, ref, D, N, L, spec, beta, kappa, lam, nmd, tau, seed, integ=OMELYAN, hot_sigma=0.8,
                 phi_sigma=0.3):
        self.lib = ref.lib
        self.h = self.lib.ref_session_create(D, N, Reference._L(L), spec.encode(), beta, kappa, lam, nmd, tau, seed,
                                             integ, hot_sigma, phi_sigma)
        if not self.h:
            raise RuntimeError("unsupported reference session configuration")

    def run(self, ntraj, series=False):
        out = np.zeros((max(ntraj, 1), 5)) if series else None
        self.lib.ref_session_run(self.h, ntraj, _d(out) if series else None)
        return out[:ntraj] if series else None

    def set_multi(self, f, mu2):
        """Install the multi-invariant potential (couplings f, one per channel; mu2), as
        hmc_higgs_multi does (src/hmc_higgs_multi.cpp:51-80)."""
        f = np.ascontiguousarray(f, np.float64)
        rc = self.lib.ref_session_set_multi(self.h, _d(f), len(f), mu2)
        if rc:
            raise RuntimeError(f"ref_session_set_multi rc={rc}")

    def set_frozen(self, on=True):
        """|phi_x| = 1 (GaugeHiggsHMC::frozen_phi) and the fields normalised, as the
        driver does under GH_FROZEN (src/hmc_higgs_multi.cpp:81-82,90)."""
        self.lib.ref_session_set_frozen(self.h, int(bool(on)))

    def acceptance(self):
        return self.lib.ref_session_acceptance(self.h)

    def close(self):
        if self.h:
            self.lib.ref_session_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def have_reference(path=REF_SO):
    return os.path.exists(path)
