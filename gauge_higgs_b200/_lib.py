"""ctypes binding of libgauge_higgs_b200.so (the C ABI of include/gauge_higgs_b200.h).

The library is the only compute path: there is no CPU fallback.  Importing this
module raises if the library has not been built, and every failing call raises
GaugeHiggsError with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libgauge_higgs_b200.so")

GH_OK = 0
ERRORS = {-1: "GH_ERR_ARG", -2: "GH_ERR_CUDA", -3: "GH_ERR_REP", -4: "GH_ERR_STATE", -5: "GH_ERR_NONFINITE",
          -6: "GH_ERR_UNSUPPORTED"}
REP_NONE, REP_FUND, REP_ADJ, REP_GENERAL = 0, 1, 2, 3
PREC_FP64, PREC_FP32_MD, PREC_FP32_ALL = 0, 1, 2
LEAPFROG, OMELYAN = 0, 1


class GaugeHiggsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class RepDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("d", C.c_int), ("real", C.c_int), ("n_boxes", C.c_int), ("dimT", C.c_long),
                ("T", C.POINTER(C.c_double)), ("W", C.POINTER(C.c_double))]


class Obs(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("H", "S_g", "S_H", "kin_P", "kin_pi", "plaquette", "L_link", "L_phi")]


class TrajRecord(C.Structure):
    _fields_ = [("dH", C.c_double), ("accepted", C.c_int), ("traj", C.c_int), ("plaquette", C.c_double),
                ("L_phi", C.c_double), ("L_link", C.c_double), ("kappa", C.c_double),
                ("beta", C.c_double)]


# numpy view of an array of TrajRecord
TRAJ_DTYPE = [("dH", "f8"), ("accepted", "i4"), ("traj", "i4"), ("plaquette", "f8"), ("L_phi", "f8"),
              ("L_link", "f8"), ("kappa", "f8"), ("beta", "f8")]


_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_u64p = C.POINTER(C.c_uint64)
_ctx = C.c_void_p

SIGNATURES = {
    "gh_set_domain": [_ctx, C.c_int, _ip, _ip, _ip, _ip],
    "gh_halo_count": [_ctx, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_longlong)],
    "gh_halo_pack": [_ctx, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "gh_halo_unpack": [_ctx, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "gh_save_fields": [_ctx],
    "gh_restore_fields": [_ctx],
    "gh_set_rep_path": [_ctx, C.c_int],
    "gh_rep_product_matrix": [C.c_int, C.POINTER(RepDesc), _dp, _dp, _ip],
    "gh_ctx_create": [C.c_int, C.c_int, C.c_int, _ip, C.POINTER(RepDesc), C.c_int, _u64p, C.POINTER(C.c_void_p)],
    "gh_ctx_destroy": [_ctx],
    "gh_set_stream": [_ctx, C.c_void_p],
    "gh_sync": [_ctx],
    "gh_info": [_ctx, _ip, _ip, _ip, _ip, _ip, _ip],
    "gh_device_bytes": [_ctx, _u64p],
    "gh_set_couplings": [_ctx, C.c_int, C.c_double, C.c_double, C.c_double],
    "gh_get_couplings": [_ctx, C.c_int, _dp, _dp, _dp],
    "gh_set_integrator": [_ctx, C.c_int, C.c_int, C.c_double],
    "gh_set_traj_count": [_ctx, C.c_int, C.c_uint64, C.c_uint64],
    "gh_get_traj_count": [_ctx, C.c_int, _u64p, _u64p, _u64p],
    "gh_set_links": [_ctx, C.c_int, _dp], "gh_get_links": [_ctx, C.c_int, _dp],
    "gh_set_mom": [_ctx, C.c_int, _dp], "gh_get_mom": [_ctx, C.c_int, _dp],
    "gh_set_phi": [_ctx, C.c_int, _dp], "gh_get_phi": [_ctx, C.c_int, _dp],
    "gh_set_pi": [_ctx, C.c_int, _dp], "gh_get_pi": [_ctx, C.c_int, _dp],
    "gh_hot_start": [_ctx, C.c_double],
    "gh_cold_start": [_ctx],
    "gh_phi_gaussian": [_ctx, C.c_uint64, C.c_double],
    "gh_phi_cold": [_ctx, C.c_double],
    "gh_mom_refresh": [_ctx, C.c_uint64],
    "gh_refresh_momenta": [_ctx],
    "gh_gauge_force": [_ctx, C.c_int, _dp],
    "gh_matter_link_force": [_ctx, C.c_int, _dp],
    "gh_scalar_force": [_ctx, C.c_int, _dp],
    "gh_kick": [_ctx, C.c_double],
    "gh_drift": [_ctx, C.c_double],
    "gh_md_evolve": [_ctx],
    "gh_reunitarize": [_ctx],
    "gh_measure": [_ctx, C.c_int, C.POINTER(Obs)],
    "gh_polyakov": [_ctx, C.c_int, C.c_int, _dp],
    "gh_trajectory": [_ctx, _dp, _ip],
    "gh_run_trajectories": [_ctx, C.c_int, C.POINTER(TrajRecord)],
    "gh_trajectory_host": [_ctx, _dp, _dp, C.POINTER(TrajRecord)],
    "gh_enqueue_trajectories": [_ctx, C.c_int],
    "gh_read_records": [_ctx, C.c_int, C.POINTER(TrajRecord)],
    "gh_use_graph": [_ctx, C.c_int],
    "gh_autotune": [_ctx, C.c_int, _dp],
    "gh_set_tile": [_ctx, C.c_int, _ip],
    "gh_get_tile": [_ctx, C.c_int, _ip],
    "gh_temper_enable": [_ctx, C.c_int, C.c_uint64],
    "gh_temper_stats": [_ctx, _u64p, _u64p, _dp],
    "gh_rep_general_info": [C.c_int, _ip, C.c_int, _ip, _ip, C.POINTER(C.c_long)],
    "gh_rep_general_build": [C.c_int, _ip, C.c_int, _dp, _dp],
    "gh_rep_path": [_ctx, _ip],
    "gh_sympow_matrix": [C.c_int, C.POINTER(RepDesc), _dp, _dp, C.POINTER(C.c_long)],
    "gh_casimir_channels": [C.c_int, C.POINTER(RepDesc), _dp, C.c_int, _ip],
    "gh_multi_superop": [C.c_int, C.POINTER(RepDesc), C.c_int, _dp, _dp],
    "gh_set_potential_multi": [_ctx, C.c_int, _dp, C.c_double],
    "gh_set_potential_quartic": [_ctx],
    "gh_set_frozen_phi": [_ctx, C.c_int],
    "gh_temper_interval": [_ctx, C.c_int],
    "gh_wilson_loop": [_ctx, C.c_int, C.c_int, C.c_int, _ip, C.c_int, _dp],
    "gh_polyakov_rep": [_ctx, C.c_int, C.c_int, _ip, C.c_int, _dp],
    "gh_normalize_phi": [_ctx],
    "gh_plaquette_noalloc": [C.c_int, C.c_int, _ip, C.c_void_p, C.c_void_p, C.c_void_p],
    "gh_mlp_create": [C.c_int, _ip, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)],
    "gh_mlp_destroy": [C.c_void_p],
    "gh_mlp_num_params": [C.c_void_p, C.POINTER(C.c_long)],
    "gh_mlp_get_params": [C.c_void_p, _fp],
    "gh_mlp_set_params": [C.c_void_p, _fp],
    "gh_mlp_grad": [C.c_void_p, _fp, _fp, C.c_int, _fp, _fp],
    "gh_mlp_adam_step": [C.c_void_p, C.c_float],
    "gh_mlp_train": [C.c_void_p, _fp, _fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64, _fp],
    "gh_mlp_predict": [C.c_void_p, _fp, C.c_int, _fp, _fp, _fp],
}


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m gauge_higgs_b200.build` "
                          "(the engine has no CPU fallback)")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.gh_rng_key.argtypes = [C.c_uint64] * 5
    lib.gh_rng_key.restype = C.c_uint64
    lib.gh_rng_uniform.argtypes = [C.c_uint64, C.c_uint64]
    lib.gh_rng_uniform.restype = C.c_double
    lib.gh_rng_gauss.argtypes = [C.c_uint64, C.c_uint64]
    lib.gh_rng_gauss.restype = C.c_double
    lib.gh_mlp_last_error.argtypes = []
    lib.gh_mlp_last_error.restype = C.c_char_p
    lib.gh_noalloc_last_error.argtypes = []
    lib.gh_noalloc_last_error.restype = C.c_char_p
    lib.gh_last_error.argtypes = [C.c_void_p]
    lib.gh_last_error.restype = C.c_char_p
    return lib


LIB = load()


def check(rc, ctx=None):
    if rc != GH_OK:
        msg = LIB.gh_last_error(ctx)
        raise GaugeHiggsError(rc, msg.decode() if msg else "")
    return rc
