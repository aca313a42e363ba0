"""What the learned surrogate gains over the method without it.

Task: locate kappa_c of the SU(2) fundamental-Higgs transition (beta = 2.3,
lambda = 0.5, 6^4; the reference's validation scan puts the chi_link peak at
kappa ~ 0.265, validation_su2higgs.dat) to +-0.005.
  * without the surrogate: a uniform batched scan at the resolution asked for
    (spacing 0.005 on [0.18, 0.34]) and the chi_link peak;
  * with it: 5 coarse points, then 3 rounds of 4 points placed by the GPU-trained
    MLP ensemble, kappa_c from the inflection of the predicted <L_link>(kappa).
Truth: a dense, high-statistics scan around the transition (not counted).
Every point is plain HMC on the GPU (batched ensembles)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_surrogate_locates_kappa_c_with_fewer_trajectories():
    from gauge_higgs_b200 import surrogate as S
    L = 6
    truth_pts, _ = S.scan(np.arange(0.245, 0.2851, 0.0025), L, ntherm=200, nmeas=4000, seed=9000)
    kc_true = S.chi_peak(truth_pts["kappa"], truth_pts["chi"])
    assert 0.25 < kc_true < 0.28            # consistent with the reference's validation scan
    kc_u, cost_u, _ = S.uniform_scan(L)
    kc_s, sd_s, cost_s, pts = S.locate_kappa_c(L)
    print(f"truth {kc_true:.4f} | uniform {kc_u:.4f} ({cost_u} traj) | surrogate {kc_s:.4f} +- {sd_s:.4f} ({cost_s} traj)")
    assert abs(kc_s - kc_true) <= 0.005
    assert cost_u >= 3 * cost_s
