"""Index arithmetic of the general-irrep slot sweep (gen_apply in
gauge_higgs_b200/csrc/gh_kernels.cuh), restated in numpy and checked exhaustively
for every tensor size the library accepts (N^n <= 200000, n <= 17).

The sweep applies U to slot k of the N^n tensor (src/rep/rep_general.hpp:184-220):
fibre f = hi * N^k + lo holds the N entries hi * N^(k+1) + lo + j * N^k.  The kernel
divides by N^k with a multiply-high by pmag[k] = ceil(2^32 / N^k) (the host table in
gh_ctx.cu), and for odd N in FP64 walks the fibres as f = lo * N^(n-1-k) + hi.  Both
walks must visit every fibre exactly once and stay inside the tensor, and the
multiply-high must equal the integer division on every fibre index it sees."""
import numpy as np
import pytest


def pmag(p):
    return ((1 << 32) + p - 1) // p


def umulhi(f, mag):
    return ((f.astype(np.uint64) * np.uint64(mag)) >> np.uint64(32)).astype(np.int64)


def sizes():
    for N in range(2, 9):
        n = 1
        while N ** n <= 200000 and n <= 17:
            yield N, n
            n += 1


@pytest.mark.parametrize("N,n", list(sizes()))
def test_both_fibre_walks_cover_the_tensor_once(N, n):
    dimT = N ** n
    nf = dimT // N
    f = np.arange(nf, dtype=np.int64)
    for k in range(n):
        blk = N ** k
        kq = n - 1 - k
        # plain walk: q = f / N^k, base = q * N^k * (N - 1) + f
        q = f if k == 0 else umulhi(f, pmag(blk))
        assert np.array_equal(q, f // blk)
        plain = q * blk * (N - 1) + f
        # outer-first walk: lo = f / N^(n-1-k), base = (f - lo * N^(n-1-k)) * N^(k+1) + lo
        lo = f if kq == 0 else umulhi(f, pmag(N ** kq))
        assert np.array_equal(lo, f // N ** kq)
        swapped = (f - lo * N ** kq) * blk * N + lo
        for base in (plain, swapped):
            assert base.min() >= 0 and base.max() + (N - 1) * blk < dimT
            entries = (base[:, None] + np.arange(N)[None, :] * blk).ravel()
            assert np.array_equal(np.sort(entries), np.arange(dimT))
        assert np.array_equal(np.sort(plain), np.sort(swapped))
