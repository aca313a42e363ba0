"""Domain-decomposed gauge + Higgs HMC driver: the counterpart of the reference's
src/mpi/gh_higgs_mpi.cpp, with its command line and output lines.

    python -m torch.distributed.run --nproc-per-node P --master-addr 127.0.0.1 \\
        -m gauge_higgs_b200.mpi_driver <rep> <L> <procgrid> <beta> <kappa> <lambda> \\
        [ntherm=40] [nmeas=80] [nmd=20] [tau=1] [seed=1]

<rep> = fund | adj | <Young rows e.g. 2,1>[:real]; <procgrid> e.g. 2,2,1,1 (its product
must equal the number of ranks, or, with one process, any grid: all subdomains then run
in this process).  One GPU per rank (LOCAL_RANK), NCCL between them.  The gauge group
is SU(GH_NCOL) (default 2, the reference build's NCOL), D = 4; GH_PRECISION=fp32 runs
FP32-MD.  The printed plaquette, L_link and L_phi do not depend on the process grid.
"""
from __future__ import annotations

import os
import sys

USAGE = ("usage: {prog} <rep> <L> <procgrid> <beta> <kappa> <lambda> [ntherm=40] [nmeas=80] [nmd=20] [tau=1] "
         "[seed=1]")


def make_rep(spec, N):
    from . import hmc as gh
    if spec == "fund":
        return gh.FundamentalRep(N)
    if spec == "adj":
        return gh.AdjointRep(N)
    real = False
    if ":" in spec:
        spec, kind = spec.split(":", 1)
        real = kind == "real"
    rows = [int(t) for t in spec.split(",") if t]
    if not rows:
        raise ValueError("bad rep spec")
    return gh.GeneralRep(N, rows, real=real)


def parse(argv):
    if len(argv) < 7:
        return None
    a = argv
    f = lambda i, d: float(a[i]) if i < len(a) else d
    n = lambda i, d: int(a[i]) if i < len(a) else d
    D = 4
    P = [1] * D
    for mu, t in enumerate([t for t in a[3].split(",") if t][:D]):
        P[mu] = int(t)
    return dict(rep=a[1], L=n(2, 8), P=P, beta=f(4, 2.3), kappa=f(5, 0.2), lam=f(6, 0.5), ntherm=n(7, 40),
                nmeas=n(8, 80), nmd=n(9, 20), tau=f(10, 1.0), seed=n(11, 1), D=D)


def main(argv=None):
    argv = sys.argv if argv is None else argv
    args = parse(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args is None:
        if rank == 0:
            print(USAGE.format(prog=argv[0]), file=sys.stderr)
        return 1
    import numpy as np
    G = [args["L"]] * args["D"]
    P = args["P"]
    prod = int(np.prod(P))
    if (world > 1 and prod != world) or any(g % p for g, p in zip(G, P)):
        if rank == 0:
            print(f"error: prod(procgrid)={prod} must equal -np={world} and divide L={args['L']}", file=sys.stderr)
        return 1
    N = int(os.environ.get("GH_NCOL", "2"))
    precision = "fp32" if os.environ.get("GH_PRECISION") == "fp32" else "fp64"
    try:
        rep = make_rep(args["rep"], N)
    except Exception as e:
        if rank == 0:
            print(f"rep error: {e}", file=sys.stderr)
        return 1
    import torch
    from .domain import DomainHMC, InProcessTransport, TorchTransport
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
        transport = TorchTransport(G, P)
    else:
        transport = InProcessTransport(G, P)
    hmc = DomainHMC(G, transport, rep=rep, N=N, seed=args["seed"], precision=precision, beta=args["beta"],
                    kappa=args["kappa"], lam=args["lam"], tau=args["tau"], nmd=args["nmd"], integ="omelyan")
    hmc.hot(0.8)
    hmc.phi_gaussian(12345, 0.3)
    m = hmc.measure()
    if rank == 0:
        print(f"# MPI gauge+Higgs: D={args['D']} SU({N}) rep={rep.name()} d={rep.d} L={args['L']}^{args['D']} "
              f"ranks={max(world, 1)} grid={'x'.join(map(str, P))}  beta={args['beta']:.3f} kappa={args['kappa']:.3f} "
              f"lambda={args['lam']:.3f} nmd={args['nmd']}")
        print(f"hot:  plaq={m['plaquette']:.10f}  L_link={m['L_link']:.10f}  L_phi={m['L_phi']:.10f}  "
              "<- identical for any procgrid")
    for _ in range(args["ntherm"]):
        hmc.trajectory()
    hmc.traj_count = 0
    hmc.accept_count = 0
    sPl = sLl = sLp = sExp = 0.0
    for _ in range(args["nmeas"]):
        hmc.trajectory()
        m = hmc.measure()
        sPl += m["plaquette"]
        sLl += m["L_link"]
        sLp += m["L_phi"]
        sExp += float(np.exp(-hmc.last_dH))
    if rank == 0:
        inv = 1.0 / max(args["nmeas"], 1)
        print(f"meas: plaq={sPl * inv:.10f}  L_link={sLl * inv:.10f}  L_phi={sLp * inv:.10f}  "
              f"({args['ntherm']}+{args['nmeas']} traj)")
        print(f"acceptance={hmc.acceptance():.4f}  <exp(-dH)>={sExp * inv:.6f}")
    hmc.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
