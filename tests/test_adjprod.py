"""General irreps through the product of adjoints (host side, gh_rep_product_matrix):
D_R(U) = Q^dag (D_adj(U) (x) ... (x) D_adj(U)) Q with the intertwiner Q the library
derives from the reference's basis W.  Pinned against the reference's own D phi and
D^dag phi (golden fixtures made by the reference: the SU(3) octet {2,1}:real and the
27-plet {4,2}:real, src/rep/rep_general.hpp:184-220) and against the oracle's tensor
construction on random links; irreps outside the product are refused."""
import numpy as np
import pytest

RNG = np.random.default_rng(5)


def su(N):
    Z = RNG.normal(size=(N, N)) + 1j * RNG.normal(size=(N, N))
    Q, R = np.linalg.qr(Z)
    Q = Q * (np.diag(R) / np.abs(np.diag(R)))
    return Q / np.linalg.det(Q) ** (1.0 / N)


def golden_rep(golden, tag):
    import gauge_higgs_b200 as gh
    reps = golden("reps")
    d, real, n, dimT, _ = reps[tag + "_info"]
    N = int(tag[1])
    rows = [int(t) for t in tag.split("_")[1].split("-")]
    return gh.GeneralRep(N, rows, real=bool(real), T=reps[tag + "_T"], W=reps[tag + "_W"]), reps


@pytest.mark.parametrize("tag,K", [("N3_2-1_real", 1), ("N3_4-2_real", 2)])
def test_product_matrix_matches_reference_rotate(golden, tag, K):
    rep, reps = golden_rep(golden, tag)
    U = reps[tag + "_U"]
    Dm, k = rep.product_matrix(U)
    assert k == K
    assert np.abs(Dm @ reps[tag + "_phi"] - reps[tag + "_rot"]).max() < 1e-12
    assert np.abs(Dm.conj().T @ reps[tag + "_phi"] - reps[tag + "_rotdag"]).max() < 1e-12


@pytest.mark.parametrize("N,rows,real", [(3, [2, 1], True), (3, [2, 1], False), (3, [4, 2], True), (3, [3, 3], False),
                                         (2, [2], False), (2, [4], False)])
def test_product_matrix_matches_tensor_construction(orc, N, rows, real):
    import gauge_higgs_b200 as gh
    from oracle.oracle import REP_GENERAL
    rep = gh.GeneralRep(N, rows, real=real)
    orep = orc.rep(REP_GENERAL, N, rep.d, int(real), rep.n_boxes, rep.dimT, rep.T, rep.W)
    for _ in range(3):
        U = su(N)
        Dm, _ = rep.product_matrix(U)
        assert np.abs(Dm - orc.rep_matrix(orep, U)).max() < 1e-12
        assert np.abs(Dm.conj().T @ Dm - np.eye(rep.d)).max() < 1e-12


@pytest.mark.parametrize("N,rows", [(3, [2]), (3, [5, 1]), (3, [3])])
def test_irreps_outside_the_product_are_refused(N, rows):
    import gauge_higgs_b200 as gh
    from gauge_higgs_b200._lib import GaugeHiggsError
    rep = gh.GeneralRep(N, rows)
    with pytest.raises(GaugeHiggsError):
        rep.product_matrix(su(N))
