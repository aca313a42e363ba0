"""Loops traced in probe irreps on the GPU (src/measure/observables.hpp:36-101): Wilson
loops W(Ra, Rb) in the fundamental (wilson_loop_fund) and in probe irreps
(wilson_loop_rep), Polyakov loops in probe irreps (polyakov_loop_rep), against the
reference on hot configurations (tests/golden/loops.npz).  The device takes the trace
as the irrep's character (Jacobi-Trudi), the reference as the trace of its
representation matrix: equal to roundoff."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [("su2_d4", 4, 2), ("su3_d4", 4, 3), ("su3_d3", 3, 3)]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "loops.npz"))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
@pytest.mark.parametrize("name,D,N", CASES)
def test_loops_match_reference(golden, name, D, N, precision, tol):
    import gauge_higgs_b200 as gh
    L = [int(x) for x in golden[name + "_L"]]
    h = gh.GaugeHMC(L, N, seed=1, precision=precision)
    h.U = golden[name + "_U"]
    specs = ["fund0", "fund", "adj", "2", "3"] + (["2,1", "1,1", "3,1"] if N == 3 else ["4", "6"])
    for spec in specs:
        rep = None if spec == "fund0" else gh.make_rep(N, spec)
        for Ra, Rb in [(1, 1), (2, 1), (2, 3)]:
            ref = float(golden[f"{name}_W_{spec}_{Ra}x{Rb}"])
            assert abs(h.wilson_loop(Ra, Rb, rep) - ref) <= tol * max(abs(ref), 0.1), (spec, Ra, Rb)
        if rep is not None:
            for tdir in range(D):
                ref = float(golden[f"{name}_P_{spec}_{tdir}"])
                assert abs(h.polyakov_loop_rep(rep, tdir) - ref) <= tol * max(abs(ref), 0.1), (spec, tdir)
    # the fundamental 1x1 loop is the average plaquette
    assert abs(h.wilson_loop(1, 1) - h.measure()["plaquette"]) < 1e-12
    h.close()


def test_bad_probe_rejected():
    import gauge_higgs_b200 as gh
    h = gh.GaugeHMC([4, 4, 4, 4], 3, seed=1)
    with pytest.raises(gh.GaugeHiggsError):
        h.wilson_loop(1, 1, [1, 2])
    with pytest.raises(gh.GaugeHiggsError):
        h.wilson_loop(0, 1)
    h.close()
