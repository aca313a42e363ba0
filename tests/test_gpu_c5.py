"""The learned coupling-scan campaign (SU(2) + fundamental Higgs, kappa_c from an MLP surrogate)
(gauge_higgs_b200/c5.py): an ensemble of five 4-128-128-128-3 MLPs over (beta, kappa,
lambda, 1/L), trained by the library's own kernels on the 64-lattice tempering batch and 12
kappas over the kappa domain at every target and size, then one active-learning round of 32 points near
the predicted chi_link peaks, each checked by 1000-trajectory plain HMC at 8^4 and
12^4.  Targets: kappa_c at two (beta, lambda) points, each at L = 8 and 12.

Without the surrogate: one uniform batched scan per target and size, kappa over the
domain [0.15, 0.35] at the asked resolution (0.005) with the same per-point statistics,
and its chi_link peak.  Truth: a dense high-statistics chi_link peak (not counted).
kappa_c of the campaign is the network's after a last fit in which each 1000-trajectory
HMC check counts four times.  The test asks for kappa_c
to +-0.005 on every target with at least 3x fewer HMC trajectories than the uniform scans.  Every point of every method is plain HMC on the
GPU; the computation is deterministic for fixed seeds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TARGETS = [(2.3, 0.5), (2.2, 0.3)]
SIZES = (8, 12)


def test_surrogate_campaign_locates_kappa_c_with_fewer_trajectories():
    from gauge_higgs_b200 import c5
    est, cost_s, data = c5.campaign(TARGETS, sizes=SIZES, seed=100)
    cost_u = 0
    rows = []
    for beta, lam in TARGETS:
        for L in SIZES:
            ku, cu, _ = c5.uniform_scan(beta, lam, L, seed=600)
            cost_u += cu
            ks, ka, _ = est[(beta, lam, L)]
            kt = c5.truth(beta, lam, L, centre=0.5 * (ks + ku))
            rows.append((beta, lam, L, kt, ks, ku))
            print(f"\nbeta {beta} lambda {lam} L {L}: truth {kt:.4f}  surrogate {ks:.4f} ({ks - kt:+.4f}; "
                  f"checks unweighted {ka:.4f})  uniform {ku:.4f} ({ku - kt:+.4f})")
    print(f"trajectories: surrogate {cost_s}, uniform scans {cost_u} ({cost_u / cost_s:.2f}x)")
    err_s = np.array([abs(r[4] - r[3]) for r in rows])
    assert cost_u >= 3 * cost_s
    assert np.all(err_s <= 0.005), err_s
