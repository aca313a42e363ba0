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
