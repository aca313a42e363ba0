"""Multi-invariant onsite potential (src/action/scalar_invariants.hpp), host side:
the channel search and the combined channel superoperator of the library, and the
oracle's V / dV/dphibar, pinned against the reference's own CasimirChannels and
MultiInvariantPotential (tests/golden/multi_potential.npz, made by
tests/golden/make_golden.py from the unmodified reference)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [(2, "fund"), (2, "adj"), (3, "fund"), (3, "adj"), (2, "6"), (3, "2"), (3, "2,1:real")]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "multi_potential.npz"))


def tag(N, spec):
    return f"N{N}_{spec.replace(',', '-').replace(':', '_')}"


@pytest.mark.parametrize("N,spec", CASES)
def test_channels_match_reference(golden, N, spec):
    import gauge_higgs_b200 as gh
    ch = gh.CasimirChannels(gh.make_rep(N, spec))
    ref = golden[tag(N, spec) + "_c2"]
    assert ch.n_channels() == len(ref)
    assert np.abs(ch.c2 - ref).max() < 1e-10


@pytest.mark.parametrize("N,spec", CASES)
def test_superop_matches_reference(golden, N, spec):
    import gauge_higgs_b200 as gh
    ch = gh.CasimirChannels(gh.make_rep(N, spec))
    t = tag(N, spec)
    A = ch.superop(golden[t + "_f"])
    ref = golden[t + "_A"]
    assert np.abs(A - ref).max() < 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("N,spec", CASES)
def test_oracle_potential_matches_reference(golden, N, spec):
    from oracle.oracle import Oracle
    O = Oracle()
    t = tag(N, spec)
    A, mu2 = golden[t + "_A"], float(golden[t + "_mu2"])
    d = int(round(np.sqrt(A.shape[0])))
    for phi, v, g in zip(golden[t + "_phi"], golden[t + "_value"], golden[t + "_dV"]):
        vo, go = O.multi_potential(d, A, mu2, phi)
        assert abs(vo - v) <= 1e-13 * abs(v)
        assert np.abs(go - g).max() <= 1e-13 * np.abs(g).max()


@pytest.mark.parametrize("name,D,N,spec", [("lat_su2_fund", 3, 2, "fund"), ("lat_su3_adj", 3, 3, "adj"),
                                           ("lat_su2_spin3", 2, 2, "6")])
def test_oracle_lattice_force_and_action(golden, name, D, N, spec):
    """The oracle's scalar force and action with the potential (superoperator from the
    library, itself pinned above) against the reference's scalar_force / scalar_action."""
    import gauge_higgs_b200 as gh
    from oracle.oracle import Oracle, OracleRep
    O = Oracle()
    rep = gh.make_rep(N, spec)
    A = gh.CasimirChannels(rep).superop(golden[name + "_f"])
    kind = {"fund": 1, "adj": 2}.get(spec, 3)
    orep = OracleRep(O.lib, kind, N, rep.d, int(rep.real), rep.n_boxes, rep.dimT, rep.T, rep.W)
    L = [int(x) for x in golden[name + "_L"]]
    U, phi = golden[name + "_U"], golden[name + "_phi"]
    F = O.scalar_force_multi(D, N, L, orep, U, phi, 0.17, A, 0.4)
    ref = golden[name + "_Fphi"]
    assert np.abs(F - ref).max() <= 1e-12 * np.abs(ref).max()
    S = O.scalar_action_multi(D, N, L, orep, U, phi, 0.17, A, 0.4)
    assert abs(S - float(golden[name + "_SH"])) <= 1e-12 * abs(float(golden[name + "_SH"]))


@pytest.mark.parametrize("N,spec", [(2, "fund"), (3, "adj"), (2, "6")])
def test_unit_couplings_give_the_square_of_phi_dag_phi(N, spec):
    """All f_c = 1: the projectors sum to the identity, so A = 2 and
    V = -mu2 phi^dag phi + (phi^dag phi)^2 (the reference driver's "auto" smoke test)."""
    import gauge_higgs_b200 as gh
    ch = gh.CasimirChannels(gh.make_rep(N, spec))
    A = ch.superop(np.ones(ch.n_channels()))
    assert np.abs(A - 2.0 * np.eye(A.shape[0])).max() < 1e-9
    pot = gh.MultiInvariantPotential(ch, np.ones(ch.n_channels()), 0.3)
    rng = np.random.default_rng(1)
    phi = rng.normal(size=ch.rep.d) + 1j * rng.normal(size=ch.rep.d)
    n2 = float(np.vdot(phi, phi).real)
    assert abs(pot.value(phi) - (-0.3 * n2 + n2 * n2)) < 1e-10 * n2 * n2


def test_coupling_count_is_checked():
    import gauge_higgs_b200 as gh
    ch = gh.CasimirChannels(gh.FundamentalRep(2))
    with pytest.raises(ValueError):
        gh.MultiInvariantPotential(ch, [1.0, 2.0, 3.0], 0.5)
    with pytest.raises(gh.GaugeHiggsError):
        ch.superop([1.0])
