"""The two-slot register path (k_gen_pair, GH_PATH_PAIR) against the tensor path and the oracle.

Irreps of two boxes that the adjoint product does not reach (SU(3) sextet {2},
antitriplet {1,1}) lift phi by the basis W to an N x N matrix Phi, apply
Phi -> U Phi U^T and project back; their matter force is 4 kappa Im Tr(T^a U Phi_y U^T
Phi_x^dag).  The same context switched to the tensor path (the reference's slot apply,
src/rep/rep_general.hpp:184-220) must give the same forces, action and MD evolution
(FP64: 1e-12 relative to the largest entry; FP32-MD: 2e-5), and the oracle's tensor
construction the same forces and action.  Lattices whose volume is not a multiple of
the 128-link work item exercise the partial last item of every direction.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.mark.parametrize("N,rows,path", [(3, [2], "pair"), (3, [1, 1], "pair"), (2, [2], "product"),
                                         (3, [2, 1], "product")])
def test_path_selection(N, rows, path):
    import gauge_higgs_b200 as gh
    h = gh.GaugeHiggsHMC([4, 4, 4, 4], gh.GeneralRep(N, rows), seed=1)
    assert h.rep_path() == path
    h.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
@pytest.mark.parametrize("N,rows,L", [(3, [2], [4, 3, 3, 5]), (3, [1, 1], [5, 3, 4, 3]), (3, [2], [6, 6, 6, 6])])
def test_pair_equals_tensor_path(N, rows, L, precision, tol):
    import gauge_higgs_b200 as gh
    rep = gh.GeneralRep(N, rows)
    out = {}
    for path in ("pair", "tensor"):
        h = gh.GaugeHiggsHMC(L, rep, seed=4, precision=precision, beta=5.7, kappa=0.12, lam=0.5, nmd=3)
        assert h.rep_path() == "pair"
        if path == "tensor":              # the path the context takes without the register form
            try:
                h.set_rep_path("tensor")
            except gh.GaugeHiggsError:
                h.set_rep_path("closed_form")
            assert h.rep_path() in ("tensor", "closed_form")
        h.hot(0.7)
        h.phi_gaussian(12345, 0.4)
        f = (h.matter_link_force(), h.scalar_force(), h.measure())
        h.refresh_momenta()
        h.md_evolve()
        out[path] = f + (h.U, h.P, h.pi, h.measure()["H"])
        h.close()
    a, b = out["pair"], out["tensor"]
    assert rel_err(a[0], b[0]) < tol
    assert rel_err(a[1], b[1]) < tol
    for k in ("S_H", "L_link"):
        assert abs(a[2][k] - b[2][k]) <= tol * max(1.0, abs(b[2][k]))
    assert rel_err(a[3], b[3]) < 10 * tol
    assert rel_err(a[4], b[4]) < 10 * tol
    assert rel_err(a[5], b[5]) < 10 * tol
    assert abs(a[6] - b[6]) <= 10 * tol * abs(b[6])


@pytest.mark.parametrize("rows,L", [([2], [3, 3, 2, 5]), ([1, 1], [4, 3, 5, 3])])
def test_pair_path_matches_oracle(orc, rows, L):
    import gauge_higgs_b200 as gh
    from oracle.oracle import REP_GENERAL
    D, N, kappa, lam = 4, 3, 0.13, 0.5
    rep = gh.GeneralRep(N, rows)
    orep = orc.rep(REP_GENERAL, N, rep.d, 0, rep.n_boxes, rep.dimT, rep.T, rep.W)
    U = orc.hot_start(D, N, L, 9, 0.7)
    phi = orc.phi_gaussian(D, L, rep.d, 9, 12345, 0, 0.5)
    h = gh.GaugeHiggsHMC(L, rep, seed=9, beta=5.7, kappa=kappa, lam=lam)
    assert h.rep_path() == "pair"
    h.U = U
    h.phi = phi
    assert rel_err(h.matter_link_force(), orc.matter_force(D, N, L, orep, U, phi, kappa)) < 1e-12
    assert rel_err(h.scalar_force(), orc.scalar_force(D, N, L, orep, U, phi, kappa, lam)) < 1e-12
    m = h.measure()
    assert abs(m["S_H"] - orc.scalar_action(D, N, L, orep, U, phi, kappa, lam)) < 1e-12 * max(1.0, abs(m["S_H"]))
    h.close()


def test_pair_switch_rejects_unavailable_paths():
    import gauge_higgs_b200 as gh
    from gauge_higgs_b200._lib import GaugeHiggsError
    h = gh.GaugeHiggsHMC([4, 4, 4, 4], gh.GeneralRep(3, [2, 1], real=True), seed=1)
    with pytest.raises(GaugeHiggsError):
        h.set_rep_path("pair")
    h.close()
    h = gh.GaugeHiggsHMC([4, 4, 4, 4], gh.GeneralRep(3, [2]), seed=1)
    with pytest.raises(GaugeHiggsError):
        h.set_rep_path("product")
    h.set_rep_path("tensor")
    h.set_rep_path("pair")
    assert h.rep_path() == "pair"
    h.close()
