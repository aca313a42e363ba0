"""The allocation-free plaquette entry point, gh_plaquette_noalloc, against the
allocating path (gh_measure).

Some callers of this library cannot allocate device memory where they measure:
a driver that records its own work into a CUDA graph (cudaMalloc is not allowed
during stream capture, cudaFree synchronises the device), or a program whose
device memory is owned by another framework's arena.  gh_plaquette_noalloc
takes their device-resident links and a device output and keeps its partial
sums in a fixed scratch array of the library.  The check runs two calls in a
row, so the second one starts from the scratch contents the first one left.
The largest case has exactly GH_NOALLOC_MAX_SITES sites, so every slot of the
scratch array is written and read.

The argument checks (sizes beyond the limit, products of extents that would
overflow, misaligned pointers) return before any CUDA call, so they run without
a GPU.
"""
import ctypes as C

import numpy as np
import pytest

MAX_SITES = 8192 * 128          # GH_NOALLOC_MAX_SITES
ALIGNED = 1 << 12               # a fake, suitably aligned device address: never dereferenced


@pytest.mark.gpu
@pytest.mark.parametrize("D,N,L", [(4, 3, [8, 6, 4, 6]), (3, 2, [6, 5, 4]), (4, 2, [16, 16, 16, 16]),
                                   (4, 2, [32, 32, 32, 32])])
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
    del U
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    Larr = (C.c_int * D)(*L)
    nplaq = int(np.prod(L)) * D * (D - 1) // 2
    for _ in range(2):
        out.fill_(-1.0)
        rc = LIB.gh_plaquette_noalloc(D, N, Larr, C.c_void_p(Ud.data_ptr()), C.c_void_p(out.data_ptr()), None)
        assert rc == 0, LIB.gh_noalloc_last_error()
        torch.cuda.synchronize()
        assert abs(float(out[1].item()) - ref) < 1e-12
        assert abs(float(out[0].item()) - ref * N * nplaq) < 1e-12 * N * nplaq
    del Ud
    torch.cuda.empty_cache()


def _call(D, N, L, U=ALIGNED, out=ALIGNED):
    from gauge_higgs_b200._lib import LIB
    Larr = (C.c_int * D)(*L)
    rc = LIB.gh_plaquette_noalloc(D, N, Larr, C.c_void_p(U), C.c_void_p(out), None)
    return rc, LIB.gh_noalloc_last_error()


def test_noalloc_rejects_oversized_lattice():
    rc, msg = _call(4, 3, [40, 40, 40, 40])           # 2.56 M sites
    assert rc == -1 and b"at most" in msg


def test_noalloc_rejects_one_site_beyond_the_limit():
    assert 17 * 61681 == MAX_SITES + 1
    rc, msg = _call(2, 2, [17, 61681])
    assert rc == -1 and b"at most" in msg
    rc, msg = _call(4, 2, [32, 32, 32, 33])
    assert rc == -1 and b"at most" in msg


def test_noalloc_rejects_extents_whose_product_overflows():
    # 2^31 - 1 per direction: the product would wrap a 64-bit count; the check refuses
    # it before multiplying
    big = 2 ** 31 - 1
    rc, msg = _call(4, 3, [big, big, big, big])
    assert rc == -1 and b"at most" in msg
    rc, msg = _call(4, 3, [65536, 65536, 65536, 65536])
    assert rc == -1 and b"at most" in msg


def test_noalloc_rejects_misaligned_pointers():
    rc, msg = _call(4, 3, [4, 4, 4, 4], U=ALIGNED + 8)
    assert rc == -1 and b"16-byte" in msg
    rc, msg = _call(4, 3, [4, 4, 4, 4], out=ALIGNED + 4)
    assert rc == -1 and b"8-byte" in msg
    rc, msg = _call(4, 3, [4, 4, 4, 4], U=0)
    assert rc == -1 and b"null" in msg
