#!/usr/bin/env python
"""Headline benchmark: SU(3) + fundamental-Higgs HMC on a 16^4 lattice,
trajectories per second, FP32-MD (FP32 fields and forces; FP64 exp(i eps P),
SU(N) projection and Hamiltonian) against the FP64 path on the same GPU, each
also end to end through the public API, with the dominant kernel's roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (beta=5.7, kappa=0.10, lambda=0.5, Omelyan nmd=16, tau=1, hot start
sigma=0.8 from Rng seed 1+rank, phi Gaussian sigma=0.3 on stream 12345): one
step = one complete HMC trajectory (momentum heatbath, H_i, 16 Omelyan steps,
H_f, Metropolis, restore on reject).  Inputs are synthetic (the reference's own
counter RNG); there is no dataset.  The L2 cache (126 MB) is flushed between
trajectories by writing a 256 MB buffer on the same stream, inside the timed
region.  Multi-GPU: one independent replica lattice per rank (the single
lattice does not shard), value = trajectories of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WL = dict(D=4, N=3, L=[16, 16, 16, 16], spec="fund", beta=5.7, kappa=0.10, lam=0.5, nmd=16, tau=1.0,
          integ="omelyan", hot_sigma=0.8, phi_sigma=0.3)
WORKLOAD = ("SU(3) + fundamental Higgs, 4D 16^4 (65536 sites), beta=5.7 kappa=0.10 lambda=0.5, "
            "Omelyan 2MN nmd=16 tau=1.0, hot start")
METRIC = "SU(3)+Higgs 16^4 trajectories/s, FP32-MD vs FP64 GPU at equal obs; % HBM peak"
# algorithmic bytes per site and launch (each field read / written once), SU(3) fundamental:
#   kick  = U 576 + phi 48 + P read+write 512 + pi read+write 96 = 1232 B (FP64), half in FP32
#   drift = P 256 + U read+write 1152 + pi 48 + phi read+write 96 = 1552 B (FP64), half in FP32
ALG_BYTES = {"kick": {"fp64": 1232, "fp32": 616}, "drift": {"fp64": 1552, "fp32": 776}}
# algorithmic flops of one kick per site, SU(3) fundamental, the reference algorithm's count
# (complex 3x3 matmul 8N^3 - 2N^2 = 198, matrix add 18, generator projection 72):
#   gauge force 4 links x (13 matmuls + 5 adds + 8 projections) = 12960, matter link force 3080,
#   scalar force 600, momentum updates 76
KICK_FLOPS_PER_SITE = 16716


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend, timeout_s=120):
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """SM clock and throttle reasons sampled during a timed region: NVML polled from a
    background thread every 2 ms (a timed region of a few tens of ms still gets samples),
    or nvidia-smi at its 100 ms minimum when NVML is not available."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.p = None
        self.thread = None

    def start(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.idx)
            self.mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            self.sm, self.reasons, self.stop_ev = [], set(), threading.Event()

            def poll():
                while not self.stop_ev.is_set():
                    self.sm.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.reasons.update(n for n, b in bits.items() if r & b)
                    self.stop_ev.wait(0.002)
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.thread is not None:
            self.stop_ev.set()
            self.thread.join(timeout=5)
            if not self.sm:
                return None
            return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": float(self.mx), "reasons": sorted(self.reasons),
                    "samples": len(self.sm), "source": "nvml"}
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(self.NAMES, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi"}


def gbps(nbytes, ms):
    """Bytes over a launch time in ms as GB/s; None when the time is not positive (a
    difference of two timings can be, e.g. under a profiler that serialises launches)."""
    return round(nbytes / (ms / 1e3) / 1e9, 1) if ms > 0 else None


def launches_per_traj(nmd, prec):
    # refresh 1 + (measure + finalize) x 2 + kicks (2 nmd + 1) + drifts 2 nmd
    # + end-of-trajectory reunitarisation (FP64 mode only) + Metropolis 1 + restore 1
    return 1 + 4 + (2 * nmd + 1) + 2 * nmd + (1 if prec == "fp64" else 0) + 2


def run_ours(a, dist):
    import torch
    torch.cuda.set_device(dist.local)
    dist.init("nccl")
    import gauge_higgs_b200 as gh

    # a dedicated stream: the engine captures its trajectory as a CUDA graph, which the
    # legacy default stream cannot host; torch work (the L2 flush) goes to the same stream
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def make(prec):
        h = gh.GaugeHiggsHMC(WL["L"], gh.FundamentalRep(WL["N"]), seed=1 + dist.rank, precision=prec,
                             beta=WL["beta"], kappa=WL["kappa"], lam=WL["lam"], nmd=WL["nmd"], tau=WL["tau"],
                             integ=WL["integ"])
        h.set_stream(stream.cuda_stream)
        h.hot(WL["hot_sigma"])
        h.phi_gaussian(12345, WL["phi_sigma"])
        if a.kick_tile:             # a fixed tile (profiling runs: timing-based choices under a profiler are not representative)
            h.set_tile([int(x) for x in a.kick_tile.split(",")])
        else:
            h.autotune(reps=3)      # kick tile shape chosen by timing (results do not depend on it)
        return h

    def timed(h, K, W, sampler=None):
        for _ in range(W):
            flush.zero_()
            h.enqueue(1)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            flush.zero_()
            h.enqueue(1)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        dist.barrier()
        ms = dist.max(e0.elapsed_time(e1))
        return ms, clocks

    def kernel_ms(h, n=40):
        """Average device time of one kick and one drift launch, back to back as in the MD
        (programmatic dependent launch overlapping each launch's tail with the next, the
        fields L2-resident as inside a trajectory): n kicks at eps = 0 (the state does not
        change), then n kick + drift pairs (the drift at the MD step); drift = pair - kick.
        CUDA events on the launching stream around each group."""
        eps = WL["tau"] / WL["nmd"]

        def group(fns):
            for _ in range(3):
                for fn, e in fns:
                    fn(e)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(n):
                for fn, e in fns:
                    fn(e)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / n

        k = group([(h.kick, 0.0)])
        pair = group([(h.kick, 0.0), (h.drift, eps)])
        return k, max(pair - k, 0.0)

    def e2e_rate(h, K):
        """End to end through the public API: gh_trajectory_host with pinned host U and phi
        copied in every trajectory, the record and (after an accepted trajectory) U and phi
        copied back."""
        U_host = torch.empty(V * 4 * 9 * 2, dtype=torch.float64, pin_memory=True).numpy()
        phi_host = torch.empty(V * 3 * 2, dtype=torch.float64, pin_memory=True).numpy()
        Uc = U_host.view(np.complex128).reshape(V, 4, 3, 3)
        pc = phi_host.view(np.complex128).reshape(V, 3)
        Uc[:] = h.U
        pc[:] = h.phi
        Ke = max(1, min(K, 50))
        for _ in range(2):
            h.trajectory_host(Uc, pc)
        torch.cuda.synchronize()
        dist.barrier()
        n_acc = 0
        t0 = time.perf_counter()
        for _ in range(Ke):
            n_acc += int(h.trajectory_host(Uc, pc).accepted)
        torch.cuda.synchronize()
        e2e_s = dist.max(time.perf_counter() - t0)
        # U and phi come back only after an accepted trajectory (a rejected one leaves the
        # host fields as they were passed in); the record (56 B) and the lattice's descriptor
        # with its trajectory counter (160 B) always
        rec_bytes = 56 + 160
        return {"value": round(dist.world * Ke / e2e_s, 3), "unit": "trajectories/s",
                "h2d_bytes_per_step": int(U_host.nbytes + phi_host.nbytes),
                "d2h_bytes_per_step": int(round(n_acc / Ke * (U_host.nbytes + phi_host.nbytes))) + rec_bytes,
                "steps": Ke, "accepted": n_acc,
                "api": "gh_trajectory_host (pinned host U, phi in; record, and U, phi when accepted, out)"}

    V = int(np.prod(WL["L"]))
    K, W = a.steps, a.warmup
    res = {}
    for prec in ("fp32", "fp64", "fp32-all"):
        h = make(prec)
        sampler = ClockSampler(dist.local) if prec == "fp32" else None
        ms, clocks = timed(h, K, W, sampler)
        recs = h.records(min(K, 1024))
        res[prec] = dict(ms=ms, clocks=clocks, acc=float(np.mean(recs["accepted"])), tile=h.get_tile(),
                         plaq=float(np.mean(recs["plaquette"])), dH=float(np.mean(recs["dH"])), h=h)
        if prec != "fp32-all":
            res[prec]["e2e"] = e2e_rate(h, K)
        res[prec]["kick_ms"], res[prec]["drift_ms"] = kernel_ms(h)

    rate = {p: dist.world * K / (res[p]["ms"] / 1e3) for p in res}
    traj_fp32, traj_fp64 = rate["fp32"], rate["fp64"]
    e2e = res["fp32"]["e2e"]

    # ---- roofline of the dominant kernel (FP32-MD path) ----
    hbm, peak_kind = peaks()
    r = res["fp32"]
    share_kick = (2 * WL["nmd"] + 1) * r["kick_ms"]
    share_drift = 2 * WL["nmd"] * r["drift_ms"]
    dom = "kick" if share_kick >= share_drift else "drift"
    dom_ms = r[dom + "_ms"]
    achieved = V * ALG_BYTES[dom]["fp32"] / (dom_ms / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic_su3_fund_16x4.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(f"{dom}_fp32_dram_bytes_per_launch")
    # the kick is arithmetic-heavy: its rate against the FP32 pipe, nominal at the sampled SM clock
    # (148 SMs x 128 FP32 lanes x 2 flop per FMA)
    clk = (r.get("clocks") or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * clk * 1e6 / 1e12
    kick_tflops = V * KICK_FLOPS_PER_SITE / (r["kick_ms"] / 1e3) / 1e12
    compute = {"kernel": "k_kick<4,3,float,FUND>", "flops_per_launch": V * KICK_FLOPS_PER_SITE,
               "achieved": round(kick_tflops, 2), "peak": round(fp32_peak, 1), "unit": "TFLOP/s",
               "frac": round(kick_tflops / fp32_peak, 4),
               "peak_source": "nominal FP32 FMA rate at the sampled SM clock (148 SMs x 128 lanes x 2)"}
    roofline = {"bound": "hbm", "kernel": "k_kick<4,3,float,FUND>" if dom == "kick" else "k_drift<3,float,double>",
                "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "peak_source": peak_kind, "traffic": traffic,
                "alg_bytes_per_launch": V * ALG_BYTES[dom]["fp32"], "avg_launch_ms": round(dom_ms, 5),
                "launch_timing": ("CUDA events around 40 back-to-back kicks (eps 0) and 40 kick + drift pairs "
                                  "(drift = pair - kick), fields L2-resident as inside a trajectory"),
                "share_of_trajectory": round((share_kick if dom == "kick" else share_drift) / (r["ms"] / K), 3),
                "fp64": {"kick_ms": round(res["fp64"]["kick_ms"], 5), "drift_ms": round(res["fp64"]["drift_ms"], 5),
                         "kick_GBps": gbps(V * ALG_BYTES["kick"]["fp64"], res["fp64"]["kick_ms"])},
                "fp32": {"kick_ms": round(r["kick_ms"], 5), "drift_ms": round(r["drift_ms"], 5),
                         "drift_GBps": gbps(V * ALG_BYTES["drift"]["fp32"], r["drift_ms"])},
                "fp32_all": {"kick_ms": round(res["fp32-all"]["kick_ms"], 5),
                             "drift_ms": round(res["fp32-all"]["drift_ms"], 5)},
                "compute": compute}

    # ---- CPU baseline: the reference itself on this host's cores (rank 0, N=1) ----
    cpu = None
    if dist.world == 1 and not a.no_cpu:
        cpu = cpu_baseline(n_traj=a.cpu_traj)

    line = {
        "metric": METRIC, "value": round(traj_fp32, 3), "unit": "trajectories/s", "n_gpus": dist.world,
        "steps": K, "warmup": W, "ms_per_step": round(res["fp32"]["ms"] / K, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (reference counter-RNG hot start and Gaussian scalar field)",
        "config": {"workload": WORKLOAD, "lattice": WL["L"], "rep": "fundamental", "beta": WL["beta"],
                   "kappa": WL["kappa"], "lambda": WL["lam"], "integrator": "omelyan", "nmd": WL["nmd"],
                   "tau": WL["tau"],
                   "precision": ("FP32-MD: FP32 fields, forces and kicks; each drift's exp(i eps P), product "
                                 "with U and Gram-Schmidt SU(N) projection in FP64; FP64 H and Metropolis"),
                   "l2": "flushed between trajectories (256 MB write, inside the timed region)",
                   "kick_tile": {"fp32": res["fp32"]["tile"], "fp64": res["fp64"]["tile"]},
                   "parallelism": f"replicas x{dist.world}"},
        "fp64": {"value": round(traj_fp64, 3), "ms_per_step": round(res["fp64"]["ms"] / K, 4),
                 "acceptance": res["fp64"]["acc"], "plaquette": res["fp64"]["plaq"], "e2e": res["fp64"]["e2e"],
                 "dtype": "f64"},
        "fp32_all": {"value": round(rate["fp32-all"], 3), "ms_per_step": round(res["fp32-all"]["ms"] / K, 4),
                     "acceptance": res["fp32-all"]["acc"], "plaquette": res["fp32-all"]["plaq"],
                     "precision": "non-default variant: the drift's exponential and projection in FP32 too"},
        "fp32_over_fp64": round(traj_fp32 / traj_fp64, 3),
        "acceptance": res["fp32"]["acc"], "plaquette": res["fp32"]["plaq"],
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": K * launches_per_traj(WL["nmd"], "fp32"),
        "clocks": res["fp32"]["clocks"],
    }
    for p in res:
        res[p]["h"].close()
    dist.close()
    if dist.rank == 0:
        print(json.dumps(line))


def cpu_baseline(n_traj=2):
    """The reference (oracle/_ref/libghref.so: the unmodified reference headers) on all
    host cores, timing its own GaugeHiggsHMC::trajectory() loop on the bench workload."""
    from oracle.oracle import Reference, RefSession, have_reference, OMELYAN
    if not have_reference():
        return cpu_baseline_port()
    ref = Reference()
    cores = ref.set_threads(os.cpu_count() or 1)
    s = RefSession(ref, WL["D"], WL["N"], WL["L"], WL["spec"], WL["beta"], WL["kappa"], WL["lam"], WL["nmd"],
                   WL["tau"], 1, OMELYAN, WL["hot_sigma"], WL["phi_sigma"])
    t0 = time.perf_counter()
    s.run(n_traj)
    dt = time.perf_counter() - t0
    s.close()
    return {"value": round(n_traj / dt, 5), "unit": "trajectories/s", "cores": cores, "kind": "reference",
            "sample": f"{n_traj} trajectories of the bench workload (setup excluded), OpenMP {cores} threads, "
                      f"{dt:.1f} s"}


def cpu_baseline_port():
    from oracle.oracle import Oracle, REP_FUND, OMELYAN
    o = Oracle()
    rep = o.rep(REP_FUND, 3)
    h = o.hmc(4, 3, WL["L"], rep, seed=1, beta=WL["beta"], kappa=WL["kappa"], lam=WL["lam"], nmd=WL["nmd"],
              integ=OMELYAN)
    h.U[:] = o.hot_start(4, 3, WL["L"], 1, 0.8)
    t0 = time.perf_counter()
    h.trajectory()
    dt = time.perf_counter() - t0
    return {"value": round(1 / dt, 5), "unit": "trajectories/s", "cores": 1, "kind": "port",
            "sample": f"1 trajectory of the bench workload on the C restatement, {dt:.1f} s"}


def run_reference(a, dist):
    """Reference arm: the reference's own CPU implementation, all host threads, rank 0 only."""
    if dist.rank != 0:
        return
    from oracle.oracle import Reference, RefSession, have_reference, OMELYAN
    if not have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libghref.so was not built"}))
        return
    ref = Reference()
    cores = ref.set_threads(os.cpu_count() or 1)
    s = RefSession(ref, WL["D"], WL["N"], WL["L"], WL["spec"], WL["beta"], WL["kappa"], WL["lam"], WL["nmd"],
                   WL["tau"], 1, OMELYAN, WL["hot_sigma"], WL["phi_sigma"])
    t0 = time.perf_counter()
    s.run(max(1, min(a.warmup, 1)))
    t_first = time.perf_counter() - t0
    # bound the whole run to a few minutes: at most ~150 s of timed trajectories
    K = max(1, min(a.steps, int(150.0 / max(t_first, 1e-3))))
    t0 = time.perf_counter()
    s.run(K)
    dt = time.perf_counter() - t0
    acc = s.acceptance()
    s.close()
    v = K / dt
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": "trajectories/s", "n_gpus": dist.world,
        "steps": K, "steps_requested": a.steps, "warmup": 1, "ms_per_step": round(dt / K * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (reference counter-RNG hot start and Gaussian scalar field)",
        "config": {"workload": WORKLOAD, "lattice": WL["L"], "rep": "fundamental", "beta": WL["beta"],
                   "kappa": WL["kappa"], "lambda": WL["lam"], "integrator": "omelyan", "nmd": WL["nmd"],
                   "tau": WL["tau"], "precision": "FP64 (reference)", "parallelism": f"OpenMP {cores} threads"},
        "acceptance": acc,
        "cpu_baseline": {"value": round(v, 5), "unit": "trajectories/s", "cores": cores, "kind": "reference",
                         "sample": f"{K} trajectories of the bench workload via GaugeHiggsHMC::trajectory()"},
        "e2e": {"value": round(v, 5), "unit": "trajectories/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_extra(a, dist):
    """Additional measurements (not the headline line): the other workloads of the benchmark
    and a lattice larger than L2.  One JSON line per case, rank 0, one GPU."""
    import torch
    torch.cuda.set_device(dist.local)
    import gauge_higgs_b200 as gh
    from oracle.oracle import Reference, RefSession, have_reference, LEAPFROG, OMELYAN
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ref = Reference() if (have_reference() and not a.no_cpu) else None
    cores = ref.set_threads(os.cpu_count() or 1) if ref else 0

    def gpu_rate(h, K, W=3):
        h.set_stream(stream.cuda_stream)
        h.autotune(reps=2)
        h.enqueue(W)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h.enqueue(K)
        e1.record(stream)
        torch.cuda.synchronize()
        rec = h.records(min(K, 1024))
        return K / (e0.elapsed_time(e1) / 1e3), rec

    def cpu_rate(D, N, L, spec, beta, kappa, lam, nmd, integ, ntraj, phi_sigma=0.3):
        if ref is None:
            return None
        s = RefSession(ref, D, N, L, spec, beta, kappa, lam, nmd, 1.0, 1, integ, 0.8, phi_sigma)
        t0 = time.perf_counter()
        s.run(ntraj)
        dt = time.perf_counter() - t0
        s.close()
        return {"value": round(ntraj / dt, 5), "cores": cores, "kind": "reference", "sample": f"{ntraj} trajectories"}

    out = []
    wl = a.workload
    if wl in ("c1", "all"):
        for prec in ("fp64", "fp32"):
            h = gh.GaugeHiggsHMC([6] * 4, gh.FundamentalRep(2), seed=1, precision=prec, beta=2.3, kappa=0.20, lam=0.5,
                                 nmd=20, integ="leapfrog")
            h.hot(0.8)
            h.phi_gaussian(12345, 0.3)
            v, rec = gpu_rate(h, 2000)
            out.append({"workload": "C1 SU(2) fund 6^4 beta=2.3 kappa=0.20 lambda=0.5 leapfrog nmd=20", "precision": prec,
                        "value": round(v, 1), "unit": "trajectories/s", "acceptance": float(rec["accepted"].mean()),
                        "cpu_baseline": cpu_rate(4, 2, [6] * 4, "fund", 2.3, 0.2, 0.5, 20, LEAPFROG, 60) if prec == "fp64" else None})
            h.close()
    if wl in ("c3", "all"):
        c3 = {"sextet": ("sextet {2}", [2], False), "octet": ("octet {2,1}:real", [2, 1], True),
              "27plet": ("27-plet {4,2}:real", [4, 2], True)}
        for spec, rows, real in (c3[k] for k in a.c3_reps.split(",")):
            rep = gh.GeneralRep(3, rows, real=real)
            for prec in ("fp64", "fp32"):
                paths = [None]
                for path in paths:
                    h = gh.GaugeHiggsHMC([12] * 4, rep, seed=1, precision=prec, beta=5.7, kappa=0.1, lam=0.5, nmd=20)
                    if path is None and h.rep_path() in ("product", "pair") and a.c3_ab:
                        paths.append("tensor")       # the same workload without the product / pair path (A/B)
                    if path is not None:
                        h.set_rep_path(path)
                    h.hot(0.8)
                    h.phi_gaussian(12345, 1.0)
                    K = 20 if (rows == [4, 2] and h.rep_path() == "tensor") else 50
                    v, rec = gpu_rate(h, K, W=1)
                    cpu = None
                    if prec == "fp64" and rows != [4, 2] and path is None:
                        sp = ",".join(map(str, rows)) + (":real" if real else "")
                        cpu = cpu_rate(4, 3, [12] * 4, sp, 5.7, 0.1, 0.5, 20, OMELYAN, 1, phi_sigma=1.0)
                    out.append({"workload": f"C3 SU(3) 12^4 {spec} beta=5.7 kappa=0.1 lambda=0.5 Omelyan nmd=20",
                                "precision": prec, "path": h.rep_path(), "value": round(v, 3), "unit": "trajectories/s",
                                "acceptance": float(rec["accepted"].mean()), "cpu_baseline": cpu})
                    h.close()
    if wl in ("c4", "all"):
        Ls = [6, 8, 10, 12]
        ext = [[L] * 4 for L in Ls for _ in range(16)]
        kap = [0.22 + 0.006 * i for _ in Ls for i in range(16)]
        seeds = list(range(1, 65))
        ens = gh.Ensemble(ext, gh.FundamentalRep(2), seeds=seeds, precision="fp32", beta=2.3, kappa=kap, lam=0.5,
                          nmd=20, integ="omelyan")
        ens.hot(0.8)
        ens.phi_gaussian(12345, 0.3)
        ens.enable_tempering(True)
        sampler = ClockSampler(dist.local)
        sampler.start()
        v, rec = gpu_rate(ens, 100)
        clocks = sampler.stop()
        att, acc, _ = ens.tempering_stats()
        # launch floor: the same trajectory graph (one lattice, same integrator, same launch
        # count) on a 2^4 lattice, where the kernels have next to no work; its time bounds what
        # removing launches (one persistent kernel) could save on the C4 ensemble
        tiny = gh.Ensemble([[2] * 4], gh.FundamentalRep(2), seeds=[1], precision="fp32", beta=2.3, kappa=0.25,
                           lam=0.5, nmd=20, integ="omelyan")
        tiny.hot(0.8)
        tiny.phi_gaussian(12345, 0.3)
        tiny.enable_tempering(True)
        v_floor, _ = gpu_rate(tiny, 400)
        tiny.close()
        sites = sum(L ** 4 for L in Ls) * 16
        cpu = None
        if ref is not None:
            t = 0.0
            for L in Ls:
                s = RefSession(ref, 4, 2, [L] * 4, "fund", 2.3, 0.25, 0.5, 20, 1.0, 1, OMELYAN, 0.8, 0.3)
                t0 = time.perf_counter()
                s.run(2)
                t += 16 * (time.perf_counter() - t0) / 2
                s.close()
            cpu = {"value": round(1.0 / t, 5), "cores": cores, "kind": "reference",
                   "sample": "2 trajectories of one lattice per L, scaled by 16 lattices per L, run serially"}
        out.append({"workload": "C4 64 SU(2)+fund lattices (16 each of L=6,8,10,12), beta=2.3 lambda=0.5, kappa grid "
                                "0.22..0.31, FP32-MD, one graph launch per ensemble trajectory, kappa tempering on",
                    "value": round(v, 2), "unit": "ensemble trajectories/s (64 lattice trajectories each)",
                    "site_updates_per_s": round(v * sites * 20 * 2, 1), "acceptance": float(rec["accepted"].mean()),
                    "swap_acceptance": float(acc.sum() / max(att.sum(), 1)), "cpu_baseline": cpu,
                    "launch_floor_ms": round(1e3 / v_floor, 4), "ms_per_ensemble_trajectory": round(1e3 / v, 4),
                    "launch_floor_share": round(v / v_floor, 4), "clocks": clocks})
        ens.close()
    if wl in ("c5", "all"):
        from gauge_higgs_b200 import c5 as C5
        targets = [tuple(float(v) for v in t.split(":")) for t in a.c5_targets.split(",")]
        sizes = tuple(int(x) for x in a.c5_sizes.split(","))
        t0 = time.perf_counter()
        est, cost_s, _ = C5.campaign(targets, sizes=sizes, seed=a.c5_seed)
        t_camp = time.perf_counter() - t0
        rows, cost_u = [], 0
        for (beta, lam) in targets:
            for L in sizes:
                ku, cu, _ = C5.uniform_scan(beta, lam, L, seed=a.c5_seed + 500)
                cost_u += cu
                kc, ks, _ = est[(beta, lam, L)]
                kt = C5.truth(beta, lam, L, centre=0.5 * (ku + kc))
                rows.append({"beta": beta, "lambda": lam, "L": L, "kappa_c_truth": round(kt, 4),
                             "surrogate": round(kc, 4), "surrogate_err": round(kc - kt, 4),
                             "surrogate_checks_unweighted": round(ks, 4), "unweighted_err": round(ks - kt, 4),
                             "uniform": round(ku, 4), "uniform_err": round(ku - kt, 4)})
        out.append({"workload": "C5 learned coupling-scan surrogate (MLP 4-128-128-128-3 x 5 over beta, kappa, lambda, "
                                "1/L; config-4 batch + 12-kappa seed lines at every target and size; 32-point active-learning round, "
                                "1000-trajectory HMC checks)", "targets": rows,
                    "trajectories_surrogate": cost_s, "trajectories_uniform": cost_u,
                    "fewer_trajectories": round(cost_u / cost_s, 2),
                    "within_0.005": {"surrogate": sum(abs(r["surrogate_err"]) <= 0.005 for r in rows),
                                     "unweighted": sum(abs(r["unweighted_err"]) <= 0.005 for r in rows),
                                     "uniform": sum(abs(r["uniform_err"]) <= 0.005 for r in rows), "of": len(rows)},
                    "campaign_s": round(t_camp, 1)})
    if wl in ("stage0", "all"):
        # the reference's SU(2) -> 2I shakedown point (scripts/su2_stage0.sh: hmc_higgs_multi with
        # rep {12}, d = 13, mu2 = 0.065 and its 13 channel couplings, beta = 2.0, nmd = 20, tau = 1)
        f2i = [0.1182, 0.0819, 0.0353, 0.0274, 0.1550, 0.0828, 0.0157, 0.0702, 0.1083, 0.1143, 0.0189, 0.1124, 0.0595]
        for Lx in [int(x) for x in a.stage0_sizes.split(",")]:
            for prec in ("fp64", "fp32"):
                rep = gh.GeneralRep(2, [12])
                # |dH| grows with the volume: at 8^4 nmd = 20 gives |dH| ~ 10 and the chain sticks,
                # so beyond 4^4 the step is halved per doubling of L (nmd = 20 L / 4), as the
                # reference's scripts raise nmd where the force gets stiff
                nmd = 20 * max(1, Lx // 4)
                h = gh.GaugeHiggsHMC([Lx] * 4, rep, seed=1, precision=prec, beta=2.0, kappa=0.1, lam=0.5, nmd=nmd)
                h.potential = gh.MultiInvariantPotential(gh.CasimirChannels(rep), f2i, 0.065)
                h.hot(0.8)
                h.phi_gaussian(12345, 0.3)
                v, rec = gpu_rate(h, 100 if Lx == 4 else 40, W=30)
                cpu = None
                if prec == "fp64" and Lx == 4 and ref is not None:
                    s = RefSession(ref, 4, 2, [Lx] * 4, "12", 2.0, 0.1, 0.5, 20, 1.0, 1, OMELYAN, 0.8, 0.3)
                    s.set_multi(f2i, 0.065)
                    s.run(1)
                    t0 = time.perf_counter()
                    s.run(3)
                    cpu = {"value": round(3 / (time.perf_counter() - t0), 5), "cores": cores, "kind": "reference",
                           "sample": "3 trajectories after one"}
                    s.close()
                out.append({"workload": f"SU(2) {{12}} (d=13) {Lx}^4, multi-invariant potential (13 channels, mu2=0.065), "
                                        f"beta=2.0 kappa=0.1, Omelyan nmd={nmd}, hot start",
                            "precision": prec,
                            "value": round(v, 2), "unit": "trajectories/s",
                            "acceptance": float(rec["accepted"].mean()), "cpu_baseline": cpu})
                h.close()
    if wl in ("scan", "all"):
        # the reference's wide (beta, kappa) phase scan of the 2I rep at 2^4 (scripts/su2_scan.sh:
        # beta 1.0..3.0 step 0.25, kappa 0.0..1.0 step 0.1, nmd by its kappa table, tau = 1), which
        # it runs as 99 single-thread jobs, nproc at a time.  Here each nmd tier is one ensemble
        # (every point a lattice of it); value = point trajectories per second over all 99 points.
        f2i = [0.1182, 0.0819, 0.0353, 0.0274, 0.1550, 0.0828, 0.0157, 0.0702, 0.1083, 0.1143, 0.0189, 0.1124, 0.0595]
        betas = [1.0 + 0.25 * i for i in range(9)]
        kappas = [0.1 * i for i in range(11)]

        def nmd_for(k):
            return 16 if k <= 0.21 else 28 if k <= 0.31 else 44 if k <= 0.51 else 56 if k <= 0.71 else 68

        tiers = {}
        for k in kappas:
            for b in betas:
                tiers.setdefault(nmd_for(k), []).append((b, k))
        for frozen, prec in ((False, "fp64"), (False, "fp32"), (True, "fp64")):
            K, total_s, acc = 20, 0.0, []
            enss = []
            for nmd, pts in sorted(tiers.items()):
                rep = gh.GeneralRep(2, [12])
                ens = gh.Ensemble([[2] * 4] * len(pts), rep, seeds=[20260602 + i for i in range(len(pts))], precision=prec,
                                  beta=[p[0] for p in pts], kappa=[p[1] for p in pts], lam=0.5, nmd=nmd,
                                  integ="omelyan")
                ens.potential = gh.MultiInvariantPotential(gh.CasimirChannels(rep), f2i, 0.065)
                ens.hot(0.8)
                ens.phi_gaussian(12345, 0.3)
                if frozen:                  # the scan under GH_FROZEN: |phi_x| = 1
                    ens.frozen_phi = True
                    ens.normalize_phi()
                v, rec = gpu_rate(ens, K, W=20)          # this tier alone
                total_s += K / v
                acc.append(float(rec["accepted"].mean()))
                enss.append(ens)
            # the tiers are independent ensembles: all of them at once, one stream each
            streams = [torch.cuda.Stream() for _ in enss]
            for ens, st in zip(enss, streams):
                ens.set_stream(st.cuda_stream)
                ens.enqueue(2)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ends = []
            for ens, st in zip(enss, streams):
                st.wait_event(e0)
                ens.enqueue(K)
                ev = torch.cuda.Event()
                ev.record(st)
                ends.append(ev)
            for ev in ends:
                stream.wait_event(ev)
            e1.record(stream)
            torch.cuda.synchronize()
            conc_s = e0.elapsed_time(e1) / 1e3
            for ens in enss:
                ens.close()
            cpu = None
            if prec == "fp64" and ref is not None:
                ref.set_threads(1)
                per_point = 0.0
                for nmd, pts in sorted(tiers.items()):
                    b, k = pts[len(pts) // 2]
                    s = RefSession(ref, 4, 2, [2] * 4, "12", b, k, 0.5, nmd, 1.0, 1, OMELYAN, 0.8, 0.3)
                    s.set_multi(f2i, 0.065)
                    s.set_frozen(frozen)
                    s.run(1)
                    t0 = time.perf_counter()
                    s.run(3)
                    per_point += len(pts) * (time.perf_counter() - t0) / 3
                    s.close()
                ref.set_threads(cores)
                cpu = {"value": round(99 * cores / per_point, 3), "cores": cores, "kind": "reference",
                       "sample": "3 trajectories of one point per nmd tier, one thread; scaled to all 99 points "
                                 f"run {cores} at a time, as the script's JOBS=nproc"}
            out.append({"workload": "2I phase scan: SU(2) {12} 2^4, multi-invariant potential, beta 1.0..3.0 x kappa "
                                    "0.0..1.0 (99 points), Omelyan nmd 16..68 by kappa, one ensemble per nmd tier"
                                    + (", frozen |phi| = 1 (GH_FROZEN)" if frozen else ""),
                        "precision": prec, "value": round(99 * K / conc_s, 1),
                        "unit": "point trajectories/s (the five tier ensembles on five streams at once)",
                        "one_tier_at_a_time": round(99 * K / total_s, 1),
                        "acceptance_by_tier": [round(x, 3) for x in acc],
                        "cpu_baseline": cpu})
    if wl in ("big", "all"):
        for prec in ("fp64", "fp32"):
            L = [32, 32, 32, 32]
            h = gh.GaugeHiggsHMC(L, gh.FundamentalRep(3), seed=1, precision=prec, beta=5.7, kappa=0.1, lam=0.5, nmd=16)
            h.set_stream(stream.cuda_stream)
            h.hot(0.8)
            h.phi_gaussian(12345, 0.3)
            h.autotune(reps=2)
            h.refresh_momenta()       # Gaussian momenta: the drift's exponential does its real work
            V = 32 ** 4
            res = {}
            for which in ("kick", "drift"):
                # the kick with eps 0 leaves P as drawn; the drift takes the Omelyan half step 1/32
                fn, eps = (h.kick, 0.0) if which == "kick" else (h.drift, 1.0 / 32)
                fn(eps)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(10):
                    fn(eps)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / 10
                res[which] = {"ms": round(ms, 4), "alg_GBps": round(V * ALG_BYTES[which][prec] / (ms / 1e3) / 1e9, 1)}
            v, _ = gpu_rate(h, 10, W=1)
            out.append({"workload": "SU(3) fund 32^4 (1,048,576 sites; fields larger than L2)", "precision": prec,
                        "value": round(v, 2), "unit": "trajectories/s", "kernels": res, "hbm_peak_GBps": peaks()[0]})
            h.close()
    if wl in ("validate", "all"):
        # FP32-MD against FP64 at equal couplings: thermalise, then n trajectories each; means
        # with 16-bin jackknife errors (src/measure/observables.hpp:129-144)
        from gauge_higgs_b200.stats import Stats
        n, ntherm = a.validate_traj, a.validate_therm
        res = {}
        for prec in ("fp64", "fp32"):
            h = gh.GaugeHiggsHMC(WL["L"], gh.FundamentalRep(3), seed=77, precision=prec, beta=WL["beta"],
                                 kappa=WL["kappa"], lam=WL["lam"], nmd=WL["nmd"], tau=WL["tau"], integ=WL["integ"])
            h.set_stream(stream.cuda_stream)
            h.hot(WL["hot_sigma"])
            h.phi_gaussian(12345, WL["phi_sigma"])
            h.run(ntherm, records=False)
            recs = []
            for t0 in range(0, n, 1000):
                recs.append(h.run(min(1000, n - t0))[:, 0])
            rec = np.concatenate(recs)
            r = {}
            for k in ("plaquette", "L_phi", "L_link", "accepted"):
                st = Stats(rec[k].astype(float))
                r[k] = (st.mean(), st.binned_error())
            st = Stats(np.exp(-rec["dH"]))
            r["exp_minus_dH"] = (st.mean(), st.binned_error())
            res[prec] = r
            h.close()
        delta = {k: round((res["fp32"][k][0] - res["fp64"][k][0]) /
                          max(np.hypot(res["fp32"][k][1], res["fp64"][k][1]), 1e-300), 2) for k in res["fp64"]}
        out.append({"workload": f"validate: FP32-MD vs FP64, {WORKLOAD}, {ntherm} thermalisation + {n} trajectories each",
                    "fp64": {k: [round(v[0], 6), round(v[1], 6)] for k, v in res["fp64"].items()},
                    "fp32": {k: [round(v[0], 6), round(v[1], 6)] for k, v in res["fp32"].items()},
                    "difference_in_combined_sigma": delta})
    for o in out:
        print(json.dumps(o))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-traj", type=int, default=10)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--stage0-sizes", default="4,8", help="lattice extents of --workload stage0 (comma list)")
    ap.add_argument("--c3-reps", default="sextet,octet,27plet", help="irreps of --workload c3 (comma list)")
    ap.add_argument("--kick-tile", default="", help="fixed kick tile (e.g. 16,2,2,2) instead of the timed choice")
    ap.add_argument("--validate-traj", type=int, default=2000)
    ap.add_argument("--validate-therm", type=int, default=200)
    ap.add_argument("--c3-ab", action="store_true", help="C3: also time product- and pair-path irreps on the tensor path")
    ap.add_argument("--c5-targets", default="2.3:0.5,2.2:0.3", help="C5: beta:lambda targets (comma list)")
    ap.add_argument("--c5-sizes", default="8,12", help="C5: lattice sizes")
    ap.add_argument("--c5-seed", type=int, default=100)
    ap.add_argument("--workload", default="c2", choices=["c2", "c1", "c3", "c4", "c5", "big", "stage0", "scan", "validate", "all"],
                    help="c2 (default) prints the headline line; the others print additional measurements")
    a = ap.parse_args()
    if a.warmup < 3 and a.impl == "ours":
        a.warmup = 3
    dist = Dist()
    if a.impl == "reference":
        run_reference(a, dist)
    elif a.workload != "c2":
        run_extra(a, dist)
    else:
        run_ours(a, dist)


if __name__ == "__main__":
    main()
