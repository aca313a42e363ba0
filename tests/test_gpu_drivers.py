"""The C++ drivers (include/gauge_higgs_b200.hpp + gauge_higgs_b200/drivers) as a
drop-in for the reference's own binaries, checked statistically against the
reference run live on the same command line.

`hmc_higgs fund 6 2.3 0.20 0.5 50 1000 20 1.0 1` (the CLI's Omelyan integrator,
src/hmc_higgs.cpp:51-54) on the GPU through the C++ driver and on the reference
(oracle/_ref, the unmodified reference headers, all host threads) with the same
arguments.  A trajectory diverges from the reference's at the ULP level (the
reference's libm is not correctly rounded), so agreement is statistical: each
observable's means differ by less than 3.5 combined jackknife errors.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "gauge_higgs_b200", "bin")
NMEAS = 1000


def parse(out):
    vals = {}
    for line in out.splitlines():
        m = re.match(r"^([^\s=]+)\s*=\s*([-+0-9.eE]+)(?:\s*\+/-\s*([-+0-9.eE]+))?", line)
        if m:
            vals[m.group(1)] = (float(m.group(2)), float(m.group(3)) if m.group(3) else None)
    return vals


@pytest.fixture(scope="module")
def ref_c1_omelyan():
    from oracle.oracle import Reference, have_reference, OMELYAN
    from gauge_higgs_b200.stats import Stats
    if not have_reference():
        pytest.fail("oracle/_ref/libghref.so (the reference harness) is not built")
    r = Reference()
    r.set_threads(os.cpu_count() or 1)
    series, acc = r.run(4, 2, [6] * 4, "fund", 2.3, 0.20, 0.5, 50, NMEAS, 20, 1.0, 1, OMELYAN)
    out = {}
    for k, col in (("plaquette", 0), ("L_phi", 1), ("L_link", 2)):
        st = Stats(series[:, col])
        out[k] = (st.mean(), st.binned_error())
    out["acceptance"] = acc
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_hmc_higgs_c1_matches_reference_statistics(precision, ref_c1_omelyan):
    env = dict(os.environ, GH_PRECISION=precision)
    r = subprocess.run([os.path.join(BIN, "hmc_higgs"), "fund", "6", "2.3", "0.20", "0.5", "50", str(NMEAS), "20",
                        "1.0", "1"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    v = parse(r.stdout)
    z = {}
    for k in ("plaquette", "L_phi", "L_link"):
        mean, err = ref_c1_omelyan[k]
        ours, oerr = v[k]
        z[k] = (ours - mean) / np.hypot(err, oerr)
    print(f"\n{precision}: deviations from the reference in combined sigma: "
          + ", ".join(f"{k} {x:+.2f}" for k, x in z.items()))
    assert all(abs(x) < 3.5 for x in z.values()), z
    assert abs(v["acceptance"][0] - ref_c1_omelyan["acceptance"]) < 0.03
    assert abs(v["<exp(-dH)>"][0] - 1.0) < 0.05
    assert v["max||UdU-I||"][0] < 1e-6


def test_gh_hmc_su3_runs():
    r = subprocess.run([os.path.join(BIN, "gh_hmc_su3"), "6", "5.7", "10", "20", "10", "1.0", "1"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    v = parse(r.stdout)
    assert 0.3 < v["plaquette"][0] < 0.7
    assert v["acceptance"][0] > 0.5


def test_driver_rejects_bad_rep():
    r = subprocess.run([os.path.join(BIN, "hmc_higgs_su3"), "1,2", "4", "5.7", "0.1", "0.5"], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1 and "rep error" in r.stderr


def test_hmc_higgs_multi_runs(tmp_path):
    """The multi-invariant potential driver (src/hmc_higgs_multi.cpp): channel listing,
    a short run with explicit couplings, its output lines and the time-series file."""
    exe = os.path.join(BIN, "hmc_higgs_multi")
    r = subprocess.run([exe, "fund"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "2 quartic channels" in r.stdout
    ts = str(tmp_path / "multi_ts.txt")
    r = subprocess.run([exe, "fund", "4", "2.3", "0.2", "1.0", "0.8,0.5", "20", "60", "16", "1.0", "3", ts],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    v = parse(r.stdout)
    assert 0.4 < v["plaquette"][0] < 0.8
    assert v["acceptance"][0] > 0.6
    assert "tau_int(L_link)" in r.stdout
    with open(ts) as f:
        assert len([ln for ln in f if not ln.startswith("#")]) == 60
    r = subprocess.run([exe, "fund", "4", "2.3", "0.2", "1.0", "1,2,3"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "need 2 couplings" in r.stderr


def test_hmc_higgs_multi_2I_scan_point():
    """One point of the reference's 2I scan (scripts/su2_scan.sh: rep {12}, 2^4, mu2 = 0.065,
    its 13 couplings, nmd 16 at kappa <= 0.21) through the driver's command line: the
    closed-form D(U) path end to end, 13 channels, a healthy acceptance."""
    exe = os.path.join(BIN, "hmc_higgs_multi")
    coup = "0.1182,0.0819,0.0353,0.0274,0.1550,0.0828,0.0157,0.0702,0.1083,0.1143,0.0189,0.1124,0.0595"
    r = subprocess.run([exe, "12", "2", "2.0", "0.1", "0.065", coup, "50", "200", "16", "1.0", "20260603"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "13 quartic channels" in r.stdout
    v = parse(r.stdout)
    assert v["acceptance"][0] > 0.8
    assert 0.0 < v["plaquette"][0] < 1.0



CPP_TEMPER = r'''
#include <cstdio>
#include "gauge_higgs_b200.hpp"
int main() {
  ghb::ReplicaTempering<4, 2> pt({4, 4, 4, 4}, ghb::FundamentalRep<2>(), {2.2, 2.25, 2.3, 2.35}, 5);
  pt.set_kappa(0.25); pt.set_lambda(0.5); pt.set_nmd(10);
  pt.hot(0.8); pt.phi_gaussian(12345, 0.3);
  for (int s = 0; s < 200; ++s) pt.step();
  for (size_t p = 0; p < pt.n_pairs(); ++p)
    std::printf("pair %zu attempts %llu accepts %llu\n", p, (unsigned long long)pt.swap_attempts(p), (unsigned long long)pt.swap_accepts(p));
  for (size_t k = 0; k < pt.n_replicas(); ++k)
    std::printf("rung %zu beta %.2f hmc_acc %.3f plaq %.6f\n", k, pt.beta(k), pt.hmc_acceptance(k), pt.measure(k).plaquette);
  return 0;
}
'''


def test_cpp_replica_tempering(tmp_path):
    """ghb::ReplicaTempering (the reference's ReplicaTempering<D,N> interface) compiled
    against include/ and the library: one swap pass per step, swaps accepted, every rung
    accepts HMC trajectories, a plaquette measured at every rung."""
    src = tmp_path / "pt.cpp"
    src.write_text(CPP_TEMPER)
    exe = tmp_path / "pt"
    lib = os.path.join(ROOT, "gauge_higgs_b200", "lib")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L" + lib, "-lgauge_higgs_b200", "-Wl,-rpath," + lib], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    pairs = [list(map(int, re.findall(r"attempts (\d+) accepts (\d+)", ln)[0])) for ln in r.stdout.splitlines()
             if ln.startswith("pair")]
    rungs = [re.findall(r"hmc_acc ([0-9.]+) plaq ([0-9.]+)", ln)[0] for ln in r.stdout.splitlines() if ln.startswith("rung")]
    assert len(pairs) == 3 and all(a == 200 and 0 < c < a for a, c in (tuple(p) for p in pairs))
    acc = [float(a) for a, _ in rungs]
    plaq = [float(p) for _, p in rungs]
    assert min(acc) > 0.5
    assert all(0.4 < p < 0.8 for p in plaq)
