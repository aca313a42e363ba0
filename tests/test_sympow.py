"""Closed-form D(U) of the single-row irreps {n} (host side, gh_sympow_matrix): the
matrix the device builds per link for large symmetric irreps, in place of the
reference's GeneralRep fast path exp(i w.T_R) (src/rep/rep_general.hpp:94-112,165-179).
Pinned against the oracle's tensor construction (src/rep/rep_general.hpp:122-131)
and the reference's own rep_matrix (its fast path where it enables one), on the
irreps of the reference's fast-path test (test/test_repfast.cpp:72-80: SU(2) {6},
{8}, {12}; SU(3) {2}, {5}) and beyond."""
import numpy as np
import pytest

from oracle.oracle import have_reference

RNG = np.random.default_rng(11)


def su(N):
    Z = RNG.normal(size=(N, N)) + 1j * RNG.normal(size=(N, N))
    Q, R = np.linalg.qr(Z)
    Q = Q * (np.diag(R) / np.abs(np.diag(R)))
    return Q / np.linalg.det(Q) ** (1.0 / N)


@pytest.mark.parametrize("N,n", [(2, 1), (2, 2), (2, 6), (2, 8), (2, 12), (2, 16), (3, 2), (3, 5), (3, 8)])
def test_closed_form_matches_tensor_construction(N, n):
    import gauge_higgs_b200 as gh
    from oracle.oracle import Oracle, REP_GENERAL
    orc = Oracle()
    rep = gh.GeneralRep(N, [n])
    orep = orc.rep(REP_GENERAL, N, rep.d, 0, rep.n_boxes, rep.dimT, rep.T, rep.W)
    for _ in range(2):
        U = su(N)
        Dc, nt = rep.closed_form_matrix(U)
        assert nt > 0
        assert np.abs(Dc - orc.rep_matrix(orep, U)).max() < 1e-12


@pytest.mark.skipif(not have_reference(), reason="reference library not built")
@pytest.mark.parametrize("N,n", [(2, 6), (2, 12), (2, 17), (3, 4), (3, 10)])
def test_closed_form_matches_reference_rep_matrix(N, n):
    """Against GeneralRep::rep_matrix: the tensor matrix, or for the large irreps the
    reference's fast path, which its self-check holds to 1e-7 of the tensor matrix."""
    import gauge_higgs_b200 as gh
    from oracle.oracle import Reference
    ref = Reference()
    rep = gh.GeneralRep(N, [n])
    info = ref.rep_info(N, str(n))
    U = su(N)
    Dc, _ = rep.closed_form_matrix(U)
    Dr = ref.rep_matrix(N, str(n), U)
    tol = 1e-9 if info["use_fast"] else 1e-12
    assert np.abs(Dc - Dr).max() < tol


def test_closed_form_is_a_unitary_homomorphism():
    """SU(2){17} (d = 18, N^n = 131072, the largest single-row SU(2) irrep under the
    reference's N^n <= 200000 cap): D(U1 U2) = D(U1) D(U2), D unitary."""
    import gauge_higgs_b200 as gh
    rep = gh.GeneralRep(2, [17])
    U1, U2 = su(2), su(2)
    D1, _ = rep.closed_form_matrix(U1)
    D2, _ = rep.closed_form_matrix(U2)
    D12, _ = rep.closed_form_matrix(U1 @ U2)
    assert np.abs(D12 - D1 @ D2).max() < 1e-11
    assert np.abs(D1 @ D1.conj().T - np.eye(rep.d)).max() < 1e-12


def test_multi_row_irrep_has_no_closed_form():
    import gauge_higgs_b200 as gh
    rep = gh.GeneralRep(3, [2, 1])
    with pytest.raises(gh.GaugeHiggsError):
        rep.closed_form_matrix(su(3))
