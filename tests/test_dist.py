"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2, 127.0.0.1).

The single lattice does not shard: N GPUs run N independent replica lattices and
the bench reduces only its timings (barrier, max over ranks).  These tests run
that plumbing as two CPU processes, and check that a rank which never reaches
the collective makes the other rank fail with an error inside the timeout
instead of hanging."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    try:
        d.init("gloo", timeout_s=5)
        if mode == "ok":
            d.barrier()
            m = d.max(float(10 * (rank + 1)))
            q.put((rank, "max", m))
        elif mode == "dead_peer":
            if rank == 1:
                q.put((rank, "left", None))
                q.close()
                q.join_thread()      # flush the message, then leave between steps
                os._exit(0)
            d.barrier()
            q.put((rank, "max", d.max(1.0)))
        d.close()
    except Exception as e:  # the surviving rank must see an error, not hang
        q.put((rank, "error", type(e).__name__))


def _run(mode, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    alive = [p for p in ps if p.is_alive()]
    for p in alive:
        p.kill()
    out = []
    while not q.empty():
        out.append(q.get())
    return out, alive


def test_replica_timing_reduction():
    out, alive = _run("ok")
    assert not alive
    maxes = sorted(v for r, k, v in out if k == "max")
    assert maxes == [20.0, 20.0]


def test_dead_rank_is_detected():
    out, alive = _run("dead_peer")
    assert not alive, "a rank hung on a collective"
    kinds = {r: k for r, k, v in out}
    assert kinds.get(1) == "left"
    assert kinds.get(0) == "error"


# ---------------------------------------------------------------------------
# replica tempering across ranks (gauge_higgs_b200/dist.py): labels and energies
# cross in one all_gather; every rank replays the same swap pass
# ---------------------------------------------------------------------------
def _temper_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime
    import numpy as np
    import torch.distributed as dist
    from gauge_higgs_b200 import dist as gd
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        ext = [[4, 4, 4, 4]] * 5 + [[6, 4, 4, 4]] * 4
        n = len(ext)
        rng = np.random.default_rng(5)
        c0 = np.concatenate([np.linspace(2.0, 2.4, 5), np.linspace(2.1, 2.4, 4)])
        steps = [rng.normal(0, 30, size=n) for _ in range(20)]
        mine = np.array_split(np.arange(n), world)[rank]
        c, counter = c0.copy(), 0
        groups = gd.ladders(ext)
        for B in steps:                       # each rank only supplies its own lattices' rows
            allv = gd.exchange(mine, np.stack([c[mine], B[mine]], 1), n)
            c, counter = gd.temper_pass(allv[:, 0], allv[:, 1], groups, counter, 0x5A7AB1EC)
        q.put((rank, c.tolist(), counter))
    finally:
        dist.destroy_process_group()


def test_cross_rank_tempering_agrees():
    """Two ranks, nine lattices in two ladders: after 20 passes both ranks hold the same
    couplings, equal to one process running the pass on all lattices."""
    import numpy as np
    sys.path.insert(0, ROOT)
    from gauge_higgs_b200 import dist as gd
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_temper_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict((r, (c, k)) for r, c, k in (q.get(timeout=120) for _ in ps))
    for p in ps:
        p.join(timeout=60)
    ext = [[4, 4, 4, 4]] * 5 + [[6, 4, 4, 4]] * 4
    rng = np.random.default_rng(5)
    c = np.concatenate([np.linspace(2.0, 2.4, 5), np.linspace(2.1, 2.4, 4)])
    steps = [rng.normal(0, 30, size=9) for _ in range(20)]
    counter = 0
    for B in steps:
        c, counter = gd.temper_pass(c, B, gd.ladders(ext), counter, 0x5A7AB1EC)
    assert res[0] == res[1]
    assert res[0][0] == c.tolist() and res[0][1] == counter
    assert sorted(c[:5]) == sorted(np.linspace(2.0, 2.4, 5))       # permutations of the ladders
