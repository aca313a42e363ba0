"""Host-side Stats against the reference's known answers (test/test_gauge.cpp:140-144)
and a numpy restatement of the block jackknife (src/measure/observables.hpp:129-144)."""
import numpy as np

from gauge_higgs_b200.stats import Stats


def test_known_series():
    s = Stats(range(1, 6))
    assert abs(s.mean() - 3.0) < 1e-12
    assert abs(s.var() - 2.0) < 1e-12
    assert abs(s.susceptibility(10.0) - 20.0) < 1e-12


def test_binned_error_and_binder():
    x = np.random.default_rng(3).normal(size=1000)
    s = Stats(x)
    bs = 1000 // 16
    bm = x[:16 * bs].reshape(16, bs).mean(1)
    assert abs(s.binned_error() - np.sqrt(bm.var(ddof=1) / 16)) < 1e-14
    d = x - x.mean()
    assert abs(s.binder() - (1 - np.mean(d ** 4) / (3 * np.mean(d ** 2) ** 2))) < 1e-12


def test_short_series_bin_rule():
    # fewer than 2 * 16 samples: the bin count drops to max(2, n // 2)
    x = np.arange(10.0) ** 1.5
    s = Stats(x)
    bm = x[:10].reshape(5, 2).mean(1)
    assert abs(s.binned_error() - np.sqrt(bm.var(ddof=1) / 5)) < 1e-13
    assert Stats([1.0]).binned_error() == 0.0
    assert Stats([]).var() == 0.0 and Stats([2.0, 2.0]).binder() == 0.0


def test_cpp_stats_agree_with_python(tmp_path):
    """ghb::Stats (the C++ mirror the drivers print with) and gauge_higgs_b200.stats give
    the same numbers."""
    import os
    import subprocess
    from conftest import ROOT
    src = tmp_path / "s.cpp"
    src.write_text('#include "gauge_higgs_b200.hpp"\n#include <cstdio>\n'
                   'int main(){ ghb::Stats s; double v; while (std::scanf("%lf", &v) == 1) s.add(v);\n'
                   ' std::printf("%.17g %.17g %.17g %.17g\\n", s.mean(), s.var(), s.binder(), s.binned_error());'
                   ' return 0; }\n')
    exe = tmp_path / "s"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    for n in (7, 40, 1000, 1003):
        x = np.random.default_rng(n).normal(size=n) * 0.1 + 0.6
        out = subprocess.run([str(exe)], input=" ".join(repr(float(v)) for v in x), capture_output=True, text=True,
                             check=True).stdout.split()
        s = Stats(x)
        for a, b in zip(map(float, out), (s.mean(), s.var(), s.binder(), s.binned_error())):
            assert abs(a - b) <= 1e-12 * max(1.0, abs(b)), (n, a, b)
