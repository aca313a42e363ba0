"""Frozen-length scalar |phi_x| = 1 on the GPU (GaugeHiggsHMC::frozen_phi,
src/hmc/gauge_higgs_hmc.hpp:38-40,61-103,133,144,172): normalize_phi, the
tangent-space momentum refresh, one kick, one geodesic drift, a whole Omelyan MD
evolution and H, each against the reference's own GaugeHiggsHMC with frozen_phi on
(tests/golden/frozen_phi.npz), and the HMC acceptance identity with the constraint."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [("su2_fund", 3, 2, "fund", 0.3), ("su3_adj", 3, 3, "adj", 0.2), ("su2_spin3", 2, 2, "6", 0.25)]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "frozen_phi.npz"))


def make(golden, name, N, spec, kappa, precision="fp64"):
    import gauge_higgs_b200 as gh
    L = [int(x) for x in golden[name + "_L"]]
    h = gh.GaugeHiggsHMC(L, gh.make_rep(N, spec), seed=3, precision=precision, beta=2.1, kappa=kappa, lam=0.5, nmd=3,
                         tau=0.5, integ="omelyan")
    h.frozen_phi = True
    h.U = golden[name + "_U0"]
    h.phi = golden[name + "_phi0"]
    return h


def close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1.0)


@pytest.mark.parametrize("name,D,N,spec,kappa", CASES)
def test_normalize_and_refresh(golden, name, D, N, spec, kappa):
    h = make(golden, name, N, spec, kappa)
    h.phi = 3.7 * golden[name + "_phi0"]
    h.normalize_phi()
    assert close(h.phi, golden[name + "_phi0"], 1e-15)
    h.refresh_momenta()
    assert close(h.P, golden[name + "_P0"], 5e-15)
    assert close(h.pi, golden[name + "_pi0"], 5e-15)
    h.close()


@pytest.mark.parametrize("name,D,N,spec,kappa", CASES)
def test_kick_drift_md_and_H(golden, name, D, N, spec, kappa):
    h = make(golden, name, N, spec, kappa)
    state = lambda: (h.__setattr__("U", golden[name + "_U0"]), h.__setattr__("phi", golden[name + "_phi0"]),
                     h.__setattr__("P", golden[name + "_P0"]), h.__setattr__("pi", golden[name + "_pi0"]))
    state()
    assert abs(h.measure()["H"] - float(golden[name + "_H0"])) <= 1e-12 * abs(float(golden[name + "_H0"]))
    h.kick(0.07)
    assert close(h.P, golden[name + "_kick_P"], 1e-12)
    assert close(h.pi, golden[name + "_kick_pi"], 1e-12)
    state()
    h.drift(0.07)
    assert close(h.U, golden[name + "_drift_U"], 1e-12)
    assert close(h.phi, golden[name + "_drift_phi"], 1e-12)
    assert close(h.pi, golden[name + "_drift_pi"], 1e-12)
    state()
    h.md_evolve()
    assert close(h.U, golden[name + "_md_U"], 1e-11)
    assert close(h.phi, golden[name + "_md_phi"], 1e-11)
    assert close(h.pi, golden[name + "_md_pi"], 1e-11)
    h.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
def test_frozen_hmc(precision, tol):
    """<exp(-dH)> = 1, a sane acceptance, and |phi_x| = 1 kept through the trajectories."""
    import gauge_higgs_b200 as gh
    h = gh.GaugeHiggsHMC([4, 4, 4, 4], gh.FundamentalRep(2), seed=41, precision=precision, beta=2.3, kappa=0.5,
                         lam=0.5, nmd=12)
    h.frozen_phi = True
    h.hot(0.4)
    h.phi_gaussian(12345, 0.6)
    h.normalize_phi()
    h.run(30, records=False)
    rec = h.run(300)[:, 0]
    mean = float(np.mean(np.exp(-rec["dH"])))
    acc = float(np.mean(rec["accepted"]))
    assert abs(mean - 1.0) < 0.12, (mean, acc)
    assert acc > 0.5, acc
    assert np.abs(np.linalg.norm(h.phi, axis=1) - 1.0).max() < tol
    assert np.abs(rec["L_phi"] - 1.0).max() < tol
    h.close()
