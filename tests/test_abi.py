"""C ABI of libgauge_higgs_b200.so without a GPU: symbols, error codes, host-side
rep construction.  No compute call here needs a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, have_gpu


def header_functions():
    txt = open(os.path.join(ROOT, "include", "gauge_higgs_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gh_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from gauge_higgs_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    names = header_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares a signature for each of them
    bound = set(_lib.SIGNATURES) | {"gh_last_error", "gh_rng_key", "gh_rng_uniform", "gh_rng_gauss",
                                      "gh_noalloc_last_error", "gh_mlp_last_error"}
    assert set(names) <= bound, set(names) - bound


def test_create_argument_errors():
    from gauge_higgs_b200._lib import LIB, RepDesc
    out = C.c_void_p()
    L = (C.c_int * 4)(4, 4, 4, 4)
    s = (C.c_uint64 * 1)(1)
    assert LIB.gh_ctx_create(5, 3, 1, L, None, 0, s, C.byref(out)) == -6
    assert b"D must be" in LIB.gh_last_error(None)
    assert LIB.gh_ctx_create(4, 7, 1, L, None, 0, s, C.byref(out)) == -6
    assert LIB.gh_ctx_create(4, 3, 0, L, None, 0, s, C.byref(out)) == -1
    assert LIB.gh_ctx_create(4, 3, 1, L, None, 9, s, C.byref(out)) == -1
    assert LIB.gh_ctx_destroy(None) == 0
    assert LIB.gh_kick(None, 0.1) == -1


@pytest.mark.skipif(have_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly():
    import gauge_higgs_b200 as gh
    with pytest.raises(gh.GaugeHiggsError, match="no CUDA device"):
        gh.GaugeHiggsHMC([4, 4, 4, 4], gh.FundamentalRep(3))


@pytest.mark.parametrize("N,spec", [(2, "2:real"), (2, "3"), (3, "1,1"), (3, "2"), (3, "2,1:real"), (3, "4,2:real")])
def test_general_rep_tables_match_reference(golden, N, spec):
    import gauge_higgs_b200 as gh
    reps = golden("reps")
    tag = f"N{N}_{spec.replace(',', '-').replace(':', '_')}"
    d, real, n, dimT, _ = reps[tag + "_info"]
    r = gh.GeneralRep.from_spec(N, spec)
    assert (r.d, int(r.real), r.n_boxes, r.dimT) == (d, real, n, dimT)
    assert np.abs(r.W - reps[tag + "_W"]).max() < 1e-13
    assert np.abs(r.T - reps[tag + "_T"]).max() < 1e-12


def test_general_rep_rejects_bad_diagrams():
    import gauge_higgs_b200 as gh
    with pytest.raises(gh.GaugeHiggsError):
        gh.GeneralRep(3, [1, 2])          # rows must be non-increasing
    with pytest.raises(gh.GaugeHiggsError):
        gh.GeneralRep(3, [1, 1, 1])       # > N-1 rows
    with pytest.raises(gh.GaugeHiggsError):
        gh.GeneralRep(2, [0])             # empty diagram


def test_symmetric_rep_su2_spin6():
    """Single-row {12} of SU(2): d = 13, N^n = 4096 (src/rep/rep_general.hpp:338-362 path)."""
    import gauge_higgs_b200 as gh
    r = gh.GeneralRep(2, [12])
    assert r.d == 13 and r.dimT == 4096
    G = r.W.conj() @ r.W.T
    assert np.abs(G - np.eye(13)).max() < 1e-12
    # Casimir: sum_a T^a T^a = C2 I with C2 = j(j+1) = 42
    C2 = sum(T @ T for T in r.T)
    assert np.abs(C2 - 42.0 * np.eye(13)).max() < 1e-9
