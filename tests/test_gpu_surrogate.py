"""What the learned surrogate gains over the method without it.

Task: locate kappa_c of the SU(2) fundamental-Higgs transition (beta = 2.3,
lambda = 0.5, 6^4; the reference's validation scan puts the chi_link peak at
kappa ~ 0.265, validation_su2higgs.dat) to +-0.005.
  * without the surrogate: a uniform batched scan at the resolution asked for
    (spacing 0.005 on [0.18, 0.34], 100 + 300 trajectories per point) and the
    chi_link peak;
  * with it: 5 coarse points, then 3 rounds of 4 points placed by the GPU-trained
    MLP ensemble (60 + 150 trajectories per point); kappa_c from the inflection of
    the predicted <L_link>(kappa), since d<L_link>/dkappa = 2 D chi_link.
Truth: a dense, high-statistics scan around the transition (not counted).
Twelve independent seeds of each method.  Every point is plain HMC on the GPU
(batched ensembles); the computation is deterministic for fixed seeds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_surrogate_locates_kappa_c_with_fewer_trajectories():
    from gauge_higgs_b200 import surrogate as S
    L = 6
    truth_pts, _ = S.scan(np.arange(0.245, 0.2851, 0.0025), L, ntherm=200, nmeas=4000, seed0=9000)
    kc_true = S.chi_peak(truth_pts["kappa"], truth_pts["chi"])
    assert 0.25 < kc_true < 0.28            # consistent with the reference's validation scan
    err_s, err_u = [], []
    for i in range(12):
        kc_s, _, cost_s, _ = S.locate_kappa_c(L, seed=100 * (i + 1))
        kc_u, cost_u, _ = S.uniform_scan(L, seed=500 + 100 * i)
        err_s.append(kc_s - kc_true)
        err_u.append(kc_u - kc_true)
    err_s, err_u = np.abs(err_s), np.abs(err_u)
    ok_s, ok_u = int(np.sum(err_s <= 0.005)), int(np.sum(err_u <= 0.005))
    print(f"truth {kc_true:.4f}; surrogate {cost_s} traj, within 0.005 in {ok_s}/12, mean |err| {err_s.mean():.4f}; "
          f"uniform {cost_u} traj, within 0.005 in {ok_u}/12, mean |err| {err_u.mean():.4f}")
    assert cost_u >= 3 * cost_s                    # at least 3x fewer trajectories ...
    assert err_s.mean() <= 0.005 and err_s.max() <= 0.01
    assert err_s.mean() <= err_u.mean()            # ... at no worse accuracy than the uniform scan
