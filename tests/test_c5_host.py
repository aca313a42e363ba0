"""Host logic of the configuration-5 campaign (gauge_higgs_b200/c5.py) without a GPU:
the seed lines cover the kappa domain at every target and size; the
active-learning choice gives every (target, size) its share of the 32 points, inside
the window around the predicted peak, at the highest member disagreement and at least
the asked spacing apart."""
import numpy as np

from gauge_higgs_b200 import c5


def test_target_lines_span_the_kappa_domain_at_every_target_and_size():
    targets, sizes = [(2.3, 0.5), (2.2, 0.3)], (8, 12)
    pts = np.array(c5.target_lines(targets, sizes, 12))
    assert len(pts) == 2 * 2 * 12
    for b, lam in targets:
        for L in sizes:
            ks = np.sort(pts[(pts[:, 0] == b) & (pts[:, 2] == lam) & (pts[:, 3] == L), 1])
            assert len(ks) == 12
            assert np.isclose(ks[0], c5.DOMAIN["kappa"][0]) and np.isclose(ks[-1], c5.DOMAIN["kappa"][1])
            assert np.allclose(np.diff(ks), np.diff(ks)[0])


class FakeSurrogate:
    """Peak at kappa = 0.2 + 0.1 (beta - 2.2) + 0.01 lambda; members disagree most at the peak."""

    def kappa_c(self, beta, lam, L, lo=0.15, hi=0.35, h=5e-4):
        return 0.2 + 0.1 * (beta - 2.2) + 0.01 * lam, 0.004

    def slope(self, beta, lam, L, grid):
        kc = self.kappa_c(beta, lam, L)[0]
        spread = np.exp(-((grid - kc) / 0.01) ** 2)
        return np.stack([spread * (1 + 0.1 * m) for m in range(5)])


def test_choose_allots_points_per_target_and_size():
    targets, sizes = [(2.3, 0.5), (2.2, 0.3), (2.4, 0.8)], (8, 12)
    pts = c5.choose(FakeSurrogate(), targets, sizes, 32)
    assert len(pts) == 32
    fs = FakeSurrogate()
    for b, lam in targets:
        kc = fs.kappa_c(b, lam, 8)[0]
        for L in sizes:
            ks = sorted(p[1] for p in pts if p[0] == b and p[2] == lam and p[3] == L)
            assert len(ks) in (5, 6)
            assert np.all(np.diff(ks) >= 0.003 - 1e-12)
            assert all(abs(k - kc) <= 0.03 + 1e-12 for k in ks)
            assert min(abs(k - kc) for k in ks) < 1e-3        # the most uncertain kappa is taken first


def test_c4_points_are_configuration_4():
    pts = np.array(c5.c4_points())
    assert len(pts) == 64
    assert sorted(set(pts[:, 3])) == [6, 8, 10, 12]
    assert np.allclose(sorted(set(np.round(pts[:, 1], 6))), 0.22 + 0.006 * np.arange(16))
    assert np.all(pts[:, 0] == 2.3) and np.all(pts[:, 2] == 0.5)


def test_weighted_repeats_only_the_checked_points():
    data = {"kappa": np.array([0.2, 0.25, 0.3]), "nmeas": np.array([150, 1000, 150]), "L": np.array([8, 8, 12])}
    w = c5.weighted(data, 1000, 4)
    assert len(w["kappa"]) == 6
    assert np.sum(w["kappa"] == 0.25) == 4 and np.sum(w["kappa"] == 0.2) == 1
