"""Replica tempering across ranks (gauge_higgs_b200/dist.py) on one GPU and one rank:
the host swap pass after every trajectory must take exactly the decisions of the
device pass of a single Ensemble (gh_temper_enable), so the records agree bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("coupling", ["beta", "kappa"])
def test_sharded_equals_device_tempering(coupling):
    import datetime
    import socket
    import torch.distributed as dist
    import gauge_higgs_b200 as gh
    from gauge_higgs_b200.dist import ShardedEnsemble
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=30))
    try:
        ext = [[4, 4, 4, 4]] * 4 + [[4, 4, 4, 6]] * 3
        seeds = list(range(11, 18))
        beta = [2.2, 2.25, 2.3, 2.35, 2.25, 2.3, 2.35] if coupling == "beta" else 2.3
        kappa = [0.22, 0.24, 0.26, 0.28, 0.24, 0.26, 0.28] if coupling == "kappa" else 0.25
        kw = dict(lam=0.5, nmd=8, precision="fp64")
        e = gh.Ensemble(ext, gh.FundamentalRep(2), seeds=seeds, beta=beta, kappa=kappa, **kw)
        e.hot(0.8)
        e.phi_gaussian(12345, 0.3)
        e.enable_tempering(True, swap_seed=0x5A7AB1EC, coupling=coupling)
        ra = e.run(60)
        att, acc, _ = e.tempering_stats()
        e.close()
        sh = ShardedEnsemble(ext, gh.FundamentalRep(2), seeds, beta, kappa, temper=coupling, **kw)
        sh.hot(0.8)
        sh.phi_gaussian(12345, 0.3)
        rb = sh.run(60)
        for k in ("dH", "accepted", "plaquette", "L_link", "kappa", "beta"):
            assert np.array_equal(ra[k], rb[k]), k
        assert [sh.stats.get(p, [0, 0])[0] for p in range(len(att))] == att.tolist()
        assert [sh.stats.get(p, [0, 0])[1] for p in range(len(acc))] == acc.tolist()
        assert acc.sum() > 0
        sh.close()
    finally:
        dist.destroy_process_group()
