"""The allocation-free plaquette entry point, gh_plaquette_noalloc, against the
allocating path (gh_measure).

Some callers of this library cannot allocate device memory where they measure:
a driver that records its own work into a CUDA graph (cudaMalloc is not allowed
during stream capture, cudaFree synchronises the device), or a program whose
device memory is owned by another framework's arena.  gh_plaquette_noalloc
takes their device-resident links and a device output and keeps its partial
sums in a fixed scratch array of the library.  The check runs two calls in a
row, so the second one starts from the scratch contents the first one left.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("D,N,L", [(4, 3, [8, 6, 4, 6]), (3, 2, [6, 5, 4]), (4, 2, [16, 16, 16, 16])])
def test_noalloc_plaquette_matches_measure(D, N, L):
    import torch
    import gauge_higgs_b200 as gh
    from gauge_higgs_b200._lib import LIB
    h = gh.GaugeHMC(L, N, seed=3)
    h.hot(0.7)
    U = h.U                                   # reference AoS layout [V, D, N, N] complex128
    ref = h.measure()["plaquette"]
    h.close()
    Ud = torch.from_numpy(np.ascontiguousarray(U).view(np.float64).ravel()).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    Larr = (C.c_int * D)(*L)
    for _ in range(2):
        out.fill_(-1.0)
        rc = LIB.gh_plaquette_noalloc(D, N, Larr, C.c_void_p(Ud.data_ptr()), C.c_void_p(out.data_ptr()), None)
        assert rc == 0, LIB.gh_noalloc_last_error()
        torch.cuda.synchronize()
        assert abs(float(out[1].item()) - ref) < 1e-12
        nplaq = np.prod(L) * D * (D - 1) // 2
        assert abs(float(out[0].item()) - ref * N * nplaq) < 1e-12 * N * nplaq


def test_noalloc_rejects_oversized_lattice():
    from gauge_higgs_b200._lib import LIB
    L = (C.c_int * 4)(40, 40, 40, 40)   # 2.56 M sites > GH_NOALLOC_MAX_SITES
    rc = LIB.gh_plaquette_noalloc(4, 3, L, C.c_void_p(1), C.c_void_p(1), None)
    assert rc == -1
    assert b"at most" in LIB.gh_noalloc_last_error()
