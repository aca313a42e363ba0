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
