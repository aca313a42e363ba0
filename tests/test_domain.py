"""Host side of the domain decomposition (gauge_higgs_b200/domain.py), no GPU: the
subdomain geometry partitions the global lattice, the global site index (the RNG key's
site) maps every interior site once, and the sequential whole-plane halo exchange
fills faces, edges and corners with the neighbours' values (src/mpi/gauge_mpi.hpp:101-139)
-- in one process and over gloo with 2 and 4 ranks.  The plane order is the one the
device's halo kernel uses (checked on the GPU in tests/test_gpu_domain.py)."""
import os

import numpy as np
import pytest

from gauge_higgs_b200.domain import InProcessTransport, Subdomain, halo_exchange, TorchTransport

GRIDS = [([4, 4, 4, 6], [1, 1, 1, 2]), ([4, 4, 4, 6], [1, 1, 2, 2]), ([6, 4, 2, 6], [2, 1, 1, 3]),
         ([4, 6, 4], [1, 2, 2])]


@pytest.mark.parametrize("G,P", GRIDS)
def test_interiors_partition_the_lattice(G, P):
    tr = InProcessTransport(G, P)
    seen = np.zeros(int(np.prod(G)), int)
    for p in tr.local_parts():
        s, g = p.interior_sites()
        assert len(s) == p.V_interior
        np.add.at(seen, g, 1)
    assert np.all(seen == 1)


def _fill(p, ncomp):
    """A field whose value at every interior site encodes its global site; NaN in halos."""
    f = np.full((p.V, ncomp), np.nan, np.complex128)
    s, g = p.interior_sites()
    f[s] = g[:, None] + 1j * np.arange(ncomp)[None, :]
    return f


def _check_all_sites(p, f, ncomp):
    g = p.global_site(np.arange(p.V))
    want = g[:, None] + 1j * np.arange(ncomp)[None, :]
    assert not np.any(np.isnan(f))
    assert np.array_equal(f, want)


@pytest.mark.parametrize("G,P", GRIDS)
def test_in_process_halo_exchange_fills_every_site(G, P):
    tr = InProcessTransport(G, P)
    parts = tr.local_parts()
    ncomp = 3
    fields = [_fill(p, ncomp) for p in parts]

    def pack(i, nu, layer):
        return fields[i][parts[i].plane_sites(nu, layer)].T.copy()      # [component][plane site]

    def unpack(i, nu, layer, buf):
        fields[i][parts[i].plane_sites(nu, layer)] = buf.T

    halo_exchange(parts, tr, pack, unpack)
    for p, f in zip(parts, fields):
        _check_all_sites(p, f, ncomp)
    assert tr.sum([1.5] * len(parts)) == 1.5 * len(parts)


def test_subdomain_rejects_uneven_grids():
    with pytest.raises(ValueError):
        Subdomain([4, 4, 4, 6], [1, 1, 1, 4], [0, 0, 0, 0])


def _gloo_worker(rank, world, port, G, P, q):
    import torch
    import torch.distributed as dist
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        tr = TorchTransport(G, P)
        p = tr.local_parts()[0]
        ncomp = 2
        f = _fill(p, ncomp)

        def pack(i, nu, layer):
            return torch.from_numpy(np.ascontiguousarray(f[p.plane_sites(nu, layer)].T))

        def unpack(i, nu, layer, buf):
            f[p.plane_sites(nu, layer)] = buf.numpy().T

        halo_exchange([p], tr, pack, unpack)
        _check_all_sites(p, f, ncomp)
        total = tr.sum([float(p.rank) + 0.25])
        q.put((rank, "ok", total))
        dist.destroy_process_group()
    except Exception as e:          # reported to the parent, which fails the test
        q.put((rank, repr(e), None))


@pytest.mark.parametrize("G,P", [([4, 4, 4, 6], [1, 1, 1, 2]), ([4, 4, 4, 6], [1, 1, 2, 2])])
def test_gloo_ranks_exchange_halos(G, P):
    import socket
    import torch.multiprocessing as mp
    world = int(np.prod(P))
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, G, P, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
    assert all(o[1] == "ok" for o in out), out
    want = sum(r + 0.25 for r in range(world))
    assert all(o[2] == want for o in out)          # every rank holds the same sum


def test_mpi_driver_argument_errors():
    """The driver's usage and process-grid checks (src/mpi/gh_higgs_mpi.cpp:35-62) need no GPU."""
    from gauge_higgs_b200 import mpi_driver
    assert mpi_driver.main(["gh_higgs_mpi", "fund", "4"]) == 1
    assert mpi_driver.main(["gh_higgs_mpi", "fund", "6", "1,1,1,4", "2.3", "0.2", "0.5"]) == 1
    assert mpi_driver.parse(["x", "fund", "8", "2,2", "2.3", "0.2", "0.5"])["P"] == [2, 2, 1, 1]
