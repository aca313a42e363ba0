"""Closed-form D(U) on the device for the large single-row irreps (k_gen_links with
the host term lists; gh_rep_path GH_PATH_CLOSED_FORM), the engine's counterpart of the
reference's GeneralRep fast path (src/rep/rep_general.hpp:94-112,165-179): which
irreps take it, forces and action against the oracle's exact tensor construction
(src/action/scalar_higgs.hpp:71-128 with src/rep/rep_general.hpp:184-220),
including irreps whose N^n tensor does not fit in shared memory, and reversibility
at the reference's SU(2) -> 2I working point (scripts/su2_stage0.sh)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F2I = [0.1182, 0.0819, 0.0353, 0.0274, 0.1550, 0.0828, 0.0157, 0.0702, 0.1083, 0.1143, 0.0189, 0.1124, 0.0595]


def test_path_selection():
    import gauge_higgs_b200 as gh
    cases = [(gh.FundamentalRep(2), "register"), (gh.GeneralRep(2, [12]), "closed_form"),
             (gh.GeneralRep(2, [17]), "closed_form"), (gh.GeneralRep(3, [8]), "closed_form"),
             (gh.GeneralRep(3, [2]), "pair"), (gh.GeneralRep(3, [2, 1]), "product")]
    for rep, path in cases:
        h = gh.GaugeHiggsHMC([2, 2, 2], rep, seed=1)
        assert h.rep_path() == path, (rep.name(), h.rep_path())
        h.close()


@pytest.mark.parametrize("N,n,L,precision,tol", [(2, 12, [3, 2, 2], "fp64", 1e-12), (2, 16, [2, 2, 2], "fp64", 1e-11),
                                                 (3, 8, [2, 2, 2], "fp64", 1e-12), (2, 12, [3, 2, 2], "fp32", 2e-5),
                                                 (3, 8, [2, 2, 2], "fp32", 2e-5)])
def test_forces_and_action_match_tensor_oracle(N, n, L, precision, tol):
    import gauge_higgs_b200 as gh
    from oracle.oracle import Oracle, REP_GENERAL
    orc = Oracle()
    rep = gh.GeneralRep(N, [n])
    D = len(L)
    h = gh.GaugeHiggsHMC(L, rep, seed=2, precision=precision, beta=2.3, kappa=0.2, lam=0.5, nmd=6)
    assert h.rep_path() == "closed_form"
    h.hot(0.6)
    h.phi_gaussian(3, 0.4)
    U, phi = h.U, h.phi
    orep = orc.rep(REP_GENERAL, N, rep.d, 0, rep.n_boxes, rep.dimT, rep.T, rep.W)
    Fm = orc.matter_force(D, N, L, orep, U, phi, 0.2)
    Fs = orc.scalar_force(D, N, L, orep, U, phi, 0.2, 0.5)
    assert np.abs(h.matter_link_force() - Fm).max() < tol * np.abs(Fm).max()
    assert np.abs(h.scalar_force() - Fs).max() < tol * np.abs(Fs).max()
    S = orc.scalar_action(D, N, L, orep, U, phi, 0.2, 0.5)
    assert abs(h.measure()["S_H"] - S) < tol * 100 * max(abs(S), 1.0)
    h.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("fp32", 2e-4)])
def test_stage0_point_reversibility(precision, tol):
    """SU(2){12} with the 13-channel multi-invariant potential at beta = 2.0, kappa = 0.6:
    forward MD, momenta flipped, MD again returns the start (test/test_scalar.cpp:122-141)."""
    import gauge_higgs_b200 as gh
    rep = gh.GeneralRep(2, [12])
    h = gh.GaugeHiggsHMC([4, 4, 4, 4], rep, seed=7, precision=precision, beta=2.0, kappa=0.6, lam=0.5, nmd=20)
    h.potential = gh.MultiInvariantPotential(gh.CasimirChannels(rep), F2I, 0.065)
    h.hot(0.8)
    h.phi_gaussian(12345, 0.3)
    h.refresh_momenta()
    U0, phi0 = h.U, h.phi
    h.md_evolve()
    h.P = -h.P
    h.pi = -h.pi
    h.md_evolve()
    assert max(np.abs(h.U - U0).max(), np.abs(h.phi - phi0).max()) < tol
    h.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_stage0_point_exp_minus_dH(precision):
    """<exp(-dH)> = 1 and the acceptance at the 2I point kappa = 0.1, nmd = 20, where the
    reference's own shakedown runs (test/test_scalar.cpp:143-156 gates)."""
    import gauge_higgs_b200 as gh
    rep = gh.GeneralRep(2, [12])
    h = gh.GaugeHiggsHMC([4, 4, 4, 4], rep, seed=3, precision=precision, beta=2.0, kappa=0.1, lam=0.5, nmd=20)
    h.potential = gh.MultiInvariantPotential(gh.CasimirChannels(rep), F2I, 0.065)
    h.hot(0.8)
    h.phi_gaussian(12345, 0.3)
    h.run(50, records=False)
    rec = h.run(300)[:, 0]
    mean = float(np.mean(np.exp(-rec["dH"])))
    acc = float(np.mean(rec["accepted"]))
    assert abs(mean - 1.0) < 0.03, (mean, acc)
    assert acc > 0.9, acc
    h.close()
