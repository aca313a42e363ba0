"""Multi-invariant onsite potential on the GPU (src/action/scalar_invariants.hpp plugged
into GaugeHiggsHMC::potential, src/hmc/gauge_higgs_hmc.hpp:25-27,108,129): the device
scalar force and action against the reference's scalar_force / scalar_action with
MultiInvariantPotential (tests/golden/multi_potential.npz), a finite-difference check
of the force, and the HMC acceptance identity <exp(-dH)> = 1 with the potential on."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
LATS = [("lat_su2_fund", 3, 2, "fund"), ("lat_su3_adj", 3, 3, "adj"), ("lat_su2_spin3", 2, 2, "6")]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "multi_potential.npz"))


def setup(golden, name, D, N, spec, precision):
    import gauge_higgs_b200 as gh
    rep = gh.make_rep(N, spec)
    L = [int(x) for x in golden[name + "_L"]]
    h = gh.GaugeHiggsHMC(L, rep, seed=5, precision=precision, beta=2.0, kappa=0.17, lam=0.5)
    h.U = golden[name + "_U"]
    h.phi = golden[name + "_phi"]
    h.potential = gh.MultiInvariantPotential(gh.CasimirChannels(rep), golden[name + "_f"], 0.4)
    return h


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
@pytest.mark.parametrize("name,D,N,spec", LATS)
def test_scalar_force_matches_reference(golden, name, D, N, spec, precision, tol):
    h = setup(golden, name, D, N, spec, precision)
    F = h.scalar_force()
    ref = golden[name + "_Fphi"]
    assert np.abs(F - ref).max() <= tol * np.abs(ref).max()
    h.close()


@pytest.mark.parametrize("name,D,N,spec", LATS)
def test_scalar_action_matches_reference(golden, name, D, N, spec):
    h = setup(golden, name, D, N, spec, "fp64")
    S = h.measure()["S_H"]
    ref = float(golden[name + "_SH"])
    assert abs(S - ref) <= 1e-12 * abs(ref)
    h.close()


def test_quartic_restored(golden):
    """potential = None gives back the quartic force bit for bit."""
    import gauge_higgs_b200 as gh
    name, D, N, spec = LATS[0]
    h = setup(golden, name, D, N, spec, "fp64")
    h.potential = None
    F0 = h.scalar_force()
    h2 = gh.GaugeHiggsHMC([int(x) for x in golden[name + "_L"]], gh.make_rep(N, spec), seed=5, beta=2.0, kappa=0.17,
                          lam=0.5)
    h2.U = golden[name + "_U"]
    h2.phi = golden[name + "_phi"]
    assert np.array_equal(F0, h2.scalar_force())
    h.close()
    h2.close()


@pytest.mark.parametrize("N,spec", [(2, "fund"), (3, "adj")])
def test_force_finite_difference(N, spec):
    """F_phi = -2 dS_H/dphi^* against central differences of the device action."""
    import gauge_higgs_b200 as gh
    rep = gh.make_rep(N, spec)
    ch = gh.CasimirChannels(rep)
    f = np.linspace(0.4, 1.3, ch.n_channels())
    h = gh.GaugeHiggsHMC([3, 3, 2], rep, seed=3, beta=2.0, kappa=0.2, lam=0.5)
    h.hot(0.5)
    h.phi_gaussian(9, 0.7)
    h.potential = gh.MultiInvariantPotential(ch, f, 0.6)
    phi0 = h.phi
    F = h.scalar_force()
    eps = 1e-5
    worst = 0.0
    for s in (0, 5, phi0.shape[0] - 1):
        for k in range(phi0.shape[1]):
            for unit in ((1.0,) if rep.real else (1.0, 1j)):
                p = phi0.copy()
                p[s, k] += eps * unit
                h.phi = p
                Sp = h.measure()["S_H"]
                p[s, k] -= 2 * eps * unit
                h.phi = p
                Sm = h.measure()["S_H"]
                fd = -(Sp - Sm) / (2 * eps)
                got = F[s, k].real if unit == 1.0 else F[s, k].imag
                worst = max(worst, abs(fd - got))
    assert worst < 1e-5
    h.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_hmc_exp_minus_dH(precision):
    """<exp(-dH)> = 1 and a sane acceptance with the multi-invariant potential on
    (the reference's acceptance gates, test/test_scalar.cpp:143-156)."""
    import gauge_higgs_b200 as gh
    rep = gh.FundamentalRep(2)
    ch = gh.CasimirChannels(rep)
    h = gh.GaugeHiggsHMC([4, 4, 4, 4], rep, seed=17, precision=precision, beta=2.3, kappa=0.2, lam=0.5, nmd=16)
    h.potential = gh.MultiInvariantPotential(ch, [0.8, 0.5], 1.0)
    h.hot(0.3)
    h.phi_gaussian(12345, 0.5)
    h.run(50, records=False)
    rec = h.run(400)[:, 0]
    mean = float(np.mean(np.exp(-rec["dH"])))
    acc = float(np.mean(rec["accepted"]))
    assert abs(mean - 1.0) < 0.12, (mean, acc)
    assert acc > 0.5, acc
    h.close()


def test_unit_couplings_reproduce_quartic_hmc():
    """f_c = 1, mu2 = 1 gives V = (phi^dag phi)^2 - phi^dag phi, the quartic potential at
    lambda = 1 up to a constant: the same seeds give the same trajectories (to roundoff)."""
    import gauge_higgs_b200 as gh
    out = []
    for multi in (False, True):
        rep = gh.FundamentalRep(2)
        h = gh.GaugeHiggsHMC([4, 4, 4, 4], rep, seed=23, beta=2.3, kappa=0.2, lam=1.0, nmd=12)
        if multi:
            ch = gh.CasimirChannels(rep)
            h.potential = gh.MultiInvariantPotential(ch, np.ones(ch.n_channels()), 1.0)
        h.hot(0.5)
        h.phi_gaussian(12345, 0.5)
        out.append(h.run(5)[:, 0])
        h.close()
    a, b = out
    assert np.array_equal(a["accepted"], b["accepted"])
    assert np.abs(a["dH"] - b["dH"]).max() < 1e-6
    assert np.abs(a["plaquette"] - b["plaquette"]).max() < 1e-9
    assert np.abs(a["L_phi"] - b["L_phi"]).max() < 1e-9


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
@pytest.mark.parametrize("N,rows,L", [(3, [2], [3, 2, 2]), (3, [2, 1], [2, 2, 2]), (2, [12], [3, 2, 2])])
def test_general_irrep_potential_vs_oracle(N, rows, L, precision, tol):
    """General irreps take w = A(M) phi from the link kernel (both of its lane layouts:
    the sextet and octet on the tensor path, SU(2){12} on the closed-form path): the
    scalar force and action against the oracle with the library's superoperator."""
    import gauge_higgs_b200 as gh
    from oracle.oracle import Oracle, OracleRep
    O = Oracle()
    rep = gh.GeneralRep(N, rows)
    ch = gh.CasimirChannels(rep)
    f = np.linspace(0.3, 1.2, ch.n_channels())
    D = len(L)
    h = gh.GaugeHiggsHMC(L, rep, seed=4, precision=precision, beta=2.0, kappa=0.17, lam=0.5)
    h.hot(0.5)
    h.phi_gaussian(7, 0.6)
    h.potential = gh.MultiInvariantPotential(ch, f, 0.4)
    U, phi = h.U, h.phi
    A = ch.superop(f)
    orep = OracleRep(O.lib, 3, N, rep.d, int(rep.real), rep.n_boxes, rep.dimT, rep.T, rep.W)
    ref = O.scalar_force_multi(D, N, L, orep, U, phi, 0.17, A, 0.4)
    assert np.abs(h.scalar_force() - ref).max() <= tol * np.abs(ref).max()
    if precision == "fp64":
        S = O.scalar_action_multi(D, N, L, orep, U, phi, 0.17, A, 0.4)
        assert abs(h.measure()["S_H"] - S) <= 1e-12 * abs(S)
    h.close()
