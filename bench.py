#!/usr/bin/env python
"""Throughput of the B200 DirectSHT forward transform (points*ell/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2] [--impl ours|reference]

A step is one forward transform (DirectSHT.__call__ semantics: polar rotation included)
of one synthetic point set already resident in HBM.  The default workload is the
survey-like single map: Nl=1024, Nx=2048, N=1e7 points with cos(theta) uniform in
[cos 1.2, cos 0.3], phi uniform in [0, 1.5 pi), lognormal(0, 0.5) weights.  Under
torchrun every rank transforms its own point set (independent requests, no collective on
the data path); the timed region is bracketed by a barrier and a device synchronise and
the slowest rank's time is reported.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as ct
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c2": dict(Nl=1024, Nx=2048, N=10_000_000, kind="c2", wkind="lognormal",
               name="survey-like single map: Nl=1024, Nx=2048, N=1e7, cos(theta)~U[cos1.2,cos0.3], "
                    "phi~U[0,1.5pi), w~lognormal(0,0.5) f64"),
    # Smaller tables for Nsight Compute captures of the same kernels (inputs still exceed L2).
    "c2prof": dict(Nl=1024, Nx=256, N=4_000_000, kind="c2", wkind="lognormal",
                   name="profiling case: Nl=1024, Nx=256, N=4e6, C2 point distribution"),
    # The sort at the full size (Nx=2048: 8188 bin keys, N=1e7) with small tables (Nl=64).
    "c2sort": dict(Nl=64, Nx=2048, N=10_000_000, kind="c2", wkind="lognormal",
                   name="sort profiling case: Nl=64, Nx=2048, N=1e7, C2 point distribution"),
    "c1": dict(Nl=256, Nx=512, N=100_000, kind="full", wkind="ones",
               name="full sky: Nl=256, Nx=512, N=1e5, cos(theta)~U[-1,1], phi~U[0,2pi), w=1 f64"),
    "c3": dict(Nl=1024, Nx=2048, N=2_000_000, kind="full", wkind="normal", maps=64,
               name="multi-map: Nl=1024, Nx=2048, N=2e6 full sky shared by 64 maps w~N(1,0.3^2) f32"),
    "c4": dict(Nl=2048, Nx=4096, N=0, kind="batch", ntrans=256, nls=(128, 256, 512, 1024, 2048),
               nrange=(1e3, 1e7),
               name="uneven batch: 256 transforms, N log-uniform [1e3,1e7], Nl in {128..2048}, Nx=2Nl, full sky, "
                    "w~U(0.5,1.5) f64; one CUDA graph, autotuned"),
    "c5": dict(Nl=2048, Nx=4096, N=0, kind="serve", nreq=64, rate=200.0, nls=(256, 512, 1024, 2048),
               nrange=(1e4, 3e7), maps=(1, 16),
               name="serving: Poisson 200 req/s, Nl in {256..2048}, Nx=2Nl, N log-uniform [1e4,3e7], 1-16 f32 maps, "
                    "caps of half-angle 0.2-pi; tables resident, HBM-budget admission, continuous batching"),
}


def make_points(spec, seed):
    rng = np.random.default_rng(seed)
    N = spec["N"]
    if spec["kind"] == "c2":
        cost = rng.uniform(np.cos(1.2), np.cos(0.3), N)
        phi = rng.uniform(0.0, 1.5 * np.pi, N)
    else:
        cost = rng.uniform(-1.0, 1.0, N)
        phi = rng.uniform(0.0, 2 * np.pi, N)
    theta = np.arccos(cost)
    if spec["wkind"] == "normal":  # float32 maps, one row per map
        w = rng.normal(1.0, 0.3, (spec.get("maps", 1), N)).astype(np.float32)
    elif spec["wkind"] == "lognormal":
        w = rng.lognormal(0.0, 0.5, N)
    elif spec["wkind"] == "uniform":
        w = rng.uniform(0.5, 1.5, N)
    else:
        w = np.ones(N)
    return theta, phi, w


# ---------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "power_w_max": max(power) if power else None}


def dram_traffic(stage, precision, N, Nlm, Nx):
    """DRAM bytes per launch of a stage's kernel from the Nsight Compute capture summarised in
    profiles/dram_traffic.json (bytes per point or per table entry), scaled to this workload."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        t = json.load(f)
    e = t.get(f"{stage}:{precision}")
    if not e:
        return None
    return e["bytes_per_point"] * N + e.get("bytes_per_table_entry", 0.0) * Nlm * Nx


def nufft_logn(Nl):
    """log2 of the NUFFT grid: 4 x 2^ceil(log2 Nl) cells, at least 128 (nufft.cu)."""
    lg = max(int(np.ceil(np.log2(max(Nl, 1)))), 0) + 2
    return max(lg, 7)


def nufft_pieces(th, ph, Nx, xmax, piece):
    """Bin pieces of a point set as the sort forms them: per (set, bin) key ceil(count/piece)."""
    c = np.cos(th)
    pol = np.abs(c) >= xmax
    x = np.where(pol, -np.sin(th) * np.cos(ph), c)
    nb = Nx - 1
    j = np.minimum((np.abs(x) * (nb / xmax)).astype(np.int64), nb - 1)
    key = (np.where(pol, 2, 0) + (x < 0)) * nb + j
    counts = np.bincount(key, minlength=4 * nb)
    return int(((counts + piece - 1) // piece).sum())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


# ---------------------------------------------------------------------------------------
def cpu_reference_run(spec, sample_n, steps, warmup, seed=0, probe_n=1000):
    """The reference's own C/OpenMP transform (csht/sht_helper.c, built into oracle/_ref) on a
    bounded sample of the workload's points, the polar/equatorial split of csht/calc_alms.py
    included.  Every timed step rotates the polar points, runs the four do_transform calls
    (polar and equatorial sets, x >= 0 and x < 0 halves) and rotates the polar alm back with
    precomputed Wigner d(pi/2) matrices (the oracle's restatement standing in for healpy's
    rotate_alm, which is absent).  Each call has a fixed cost independent of the points (it
    zeroes one 4 Nl Nx accumulator per thread and contracts every (l, m) over all nodes), so
    the run also times `probe_n`-point steps for that fixed part and splits the step time into
    fixed + per-point costs, from which the throughput at the workload's full N follows."""
    from oracle import dsht_oracle as O
    from oracle import ref_csht
    if not ref_csht.available():
        return None
    Nl, Nx, N_full = spec["Nl"], spec["Nx"], spec["N"]
    t0 = time.time()
    ref = ref_csht.RefCSHT(Nl, Nx)
    t_tables = time.time() - t0
    t0 = time.time()
    rot = O.AlmRotator(Nl)
    t_dmat = time.time() - t0

    def points(n, sd):
        th, ph, w = make_points(dict(spec, N=n), sd)
        if w.ndim == 2:  # the reference transforms one map per call; time the first
            w = np.ascontiguousarray(w[0], dtype=np.float64)
        return th, ph, w

    def one_step(th, ph, w):
        t0 = time.perf_counter()
        pol = np.abs(np.cos(th)) >= 0.75
        alm = np.zeros(ref.Nlm, dtype=np.complex128)
        if pol.any():
            tr, pr = O.rotate_points(th[pol], ph[pol])
            alm += rot(ref.basic(tr, pr, w[pol]))
        equ = ~pol
        if equ.any():
            alm += ref.basic(th[equ], ph[equ], w[equ])
        return time.perf_counter() - t0

    probe = points(probe_n, seed + 999)
    sample = points(sample_n, seed + 1000)
    # Warm-up and fixed-cost probe: the CPU path has no state to warm beyond paging in its
    # tables, so the W warm-up steps run the probe-sized sample and time the fixed part.
    fixed = [one_step(*probe) for _ in range(max(warmup, 1))]
    times = [one_step(*sample) for _ in range(steps)]
    sec = float(np.mean(times))
    t_fixed = float(np.median(fixed))
    per_point = max(sec - t_fixed, 0.0) / sample_n
    # a split is only resolved when the sample step clearly exceeds the fixed part (the probe
    # steps' noise is a few percent of the fixed part)
    resolved = sec > 1.05 * t_fixed
    t_full = t_fixed + per_point * N_full if (N_full and resolved) else None
    return {"value": sample_n * Nl / sec, "unit": "points*ell/s", "cores": os.cpu_count(),
            "kind": "reference", "seconds_per_step": sec, "table_build_s": t_tables, "dmatrix_build_s": t_dmat,
            "sample_points": sample_n, "same_config": sample_n == N_full,
            "split": {"fixed_s_per_step": t_fixed, "per_point_s": per_point,
                      "probe": f"{max(warmup, 1)} steps of {probe_n} points (the warm-up steps)",
                      "note": "fixed = four do_transform calls and the alm rotation at ~no points",
                      "resolved": resolved},
            "at_config": None if t_full is None else {
                "N": N_full, "seconds_per_transform": t_full, "value": N_full * Nl / t_full,
                "how": "fixed + per_point x N from this run's split (extrapolated, not timed)"},
            "sample": f"{sample_n} points of the same distribution (one map) per step through "
                      f"csht/sht_helper.c do_transform (OpenMP, {os.cpu_count()} threads) at Nl={Nl}, Nx={Nx}, "
                      f"polar point and alm rotations inside the timed region"}


def run_reference_arm(args, spec):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    r = cpu_reference_run(spec, args.ref_sample, args.steps, args.warmup)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/sht_helper.so (csht) not built"}))
        return 0
    line = {"metric": "points*ell/s", "value": r["value"], "unit": "points*ell/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["seconds_per_step"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": spec["name"], "Nl": spec["Nl"], "Nx": spec["Nx"], "N": args.ref_sample,
                       "N_workload": spec["N"], "same_config": r["same_config"],
                       "maps": 1, "maps_note": "points*ell/s counts point x map x ell; one map per call"},
            "cpu_baseline": {"value": r["value"], "unit": r["unit"], "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "split": r["split"], "at_config": r["at_config"],
            "caveat": None if r["same_config"] else (
                f"each step transforms {args.ref_sample} of the workload's {spec['N']} points (a full-size step "
                f"takes minutes on the host); per-call fixed costs weigh more at this size, so the value "
                f"understates the reference at the full N -- at_config gives the split-based estimate"),
            "e2e": {"value": r["value"], "unit": "points*ell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
def _dist_setup():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    return world, rank, local, dev


def batch_transforms(spec, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(spec["ntrans"]):
        Nl = int(rng.choice(spec["nls"]))
        N = int(np.exp(rng.uniform(np.log(spec["nrange"][0]), np.log(spec["nrange"][1]))))
        th = np.arccos(rng.uniform(-1, 1, N))
        ph = rng.uniform(0, 2 * np.pi, N)
        w = rng.uniform(0.5, 1.5, N)
        out.append((Nl, 2 * Nl, th, ph, w))
    return out


def run_batch(args, spec):
    """The uneven batch: every rank runs its own 256 transforms (replicas), captured once in
    a CUDA graph; a step is one graph launch over the whole batch."""
    import torch
    from directsht_b200 import _lib as L
    from directsht_b200.batch import PlanCache, TransformBatch, autotune
    from directsht_b200.dist import reduce_scalar
    world, rank, local, dev = _dist_setup()
    lib = L.load()
    ts = batch_transforms(spec, seed=rank)
    t0 = time.time()
    cache = PlanCache(device=dev, precision="mixed", compact_min_nl=1024)
    for Nl in spec["nls"]:
        cache.get(Nl, 2 * Nl)
    t_plans = time.time() - t0
    b = TransformBatch(cache, ts)
    t0 = time.time()
    cfg = autotune(b, path=args.tune_cache, reps=1)
    t_tune = time.time() - t0
    b.capture()
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        b.run()
    torch.cuda.synchronize()
    b.check()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = lib.dsht_launch_count()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev[0].record(stream)
    for k in range(args.steps):
        b.run()
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    per_step = np.array([ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)])
    total_ms = reduce_scalar(ev[0].elapsed_time(ev[-1]), "max", dev)
    ms_step = total_ms / args.steps
    pe = b.points_ell()
    # graph replays launch no kernels from the host: count one eager run's launches instead
    b.release()
    l0 = lib.dsht_launch_count()
    b.run()
    torch.cuda.synchronize()
    launches = lib.dsht_launch_count() - l0
    # each (Nl, Nx) group alone, eager, with its tuned configuration (where the time goes)
    group_ms = {}
    for key in b.groups:
        sub = TransformBatch.__new__(TransformBatch)
        sub.__dict__.update(b.__dict__)
        sub.groups = {key: b.groups[key]}
        sub.config = {key: b.config[key]}
        sub.graph = None
        sub._build()
        sub.run()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        sub.run()
        g1.record(stream)
        torch.cuda.synchronize()
        group_ms[f"{key[0]}x{key[1]}"] = g0.elapsed_time(g1)
        del sub
    # accuracy of a sample against FP64 plans (Nl <= 512, whose FP64 tables fit beside the rest)
    fp64 = PlanCache(device=dev, precision="fp64")
    errs = []
    for i, t in enumerate(ts):
        if t[0] <= 512 and len(errs) < 24:
            ref = fp64.get(t[0], t[1])(t[2], t[3], t[4])
            errs.append(float(np.abs(b.alms[i].cpu().numpy() - ref).max() / np.abs(ref).max()))
    # end to end: inputs from pinned host memory every step, alm back to pinned host memory
    e2e = None
    if args.e2e_steps > 0:
        hp = [[torch.from_numpy(a).pin_memory() for a in t[2:5]] for t in ts]
        outs = [torch.empty_like(a, device="cpu").pin_memory() for a in b.alms]
        h2d = sum(a.numel() * 8 for h in hp for a in h)
        d2h = sum(a.numel() * 16 for a in b.alms)

        def e2e_step():
            for h, th_, ph_, w_ in zip(hp, b.thetas, b.phis, b.ws_):
                th_.copy_(h[0], non_blocking=True)
                ph_.copy_(h[1], non_blocking=True)
                w_.copy_(h[2], non_blocking=True)
            b.run()
            for o, a in zip(outs, b.alms):
                o.copy_(a, non_blocking=True)
            torch.cuda.synchronize()
        e2e_step()
        tt = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        e2e_s = reduce_scalar((time.perf_counter() - tt) / args.e2e_steps, "max", dev)
        e2e = {"value": world * pe / e2e_s, "unit": "points*ell/s", "ms_per_step": e2e_s * 1e3,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "path": "pinned host -> device copies of all 256 point sets, eager batch run (dsht_enqueue_batch), "
                       "all alm -> pinned host; wall clock"}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        groups = {f"{k[0]}x{k[1]}": {"transforms": len(v), "points": int(sum(b.Ns[i] for i in v)),
                                       "config": cfg.get(k), "ms_alone": group_ms.get(f"{k[0]}x{k[1]}")}
                  for k, v in b.groups.items()}
        line = {"metric": "points*ell/s", "value": world * pe / (ms_step / 1e3), "unit": "points*ell/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64 NUFFT, i8 tensor-core or f64 direct bin sums (AUTO) + i8 digit-table contraction + f64", "data": "synthetic",
                "config": {"workload": spec["name"], "transforms": len(ts), "points": int(sum(b.Ns)),
                           "points_ell": pe, "precision": "mixed (compact digit tables only for Nl >= 1024)",
                           "l2": "inputs (GBs) and tables (79 GB) exceed L2", "parallelism": f"replicas x{world}",
                           "groups": groups},
                "p50_ms": float(np.percentile(per_step, 50)), "p99_ms": float(np.percentile(per_step, 99)),
                "plan_build_s": t_plans, "autotune_s": t_tune, "max_rel_err_vs_fp64_sample": max(errs) if errs else None,
                "e2e": e2e, "gpu_launches": int(launches), "clocks": clk,
                "note": "a step is one CUDA-graph launch of the whole batch; gpu_launches counts one eager run"}
        print(json.dumps(line), flush=True)
    return 0


def run_serve(args, spec):
    """The serving stream: Poisson arrivals replayed in wall-clock time into the request
    loop; throughput over the makespan and latency submit -> alm in host memory."""
    import torch
    from directsht_b200 import _lib as L
    from directsht_b200.batch import PlanCache
    from directsht_b200.dist import reduce_scalar
    from directsht_b200.serve import GpuExecutor, Server, poisson_requests, replay
    world, rank, local, dev = _dist_setup()
    lib = L.load()
    t0 = time.time()
    cache = PlanCache(device=dev, precision="mixed", compact_min_nl=1024)
    for Nl in spec["nls"]:
        cache.get(Nl, 2 * Nl)
    t_plans = time.time() - t0
    free, total = torch.cuda.mem_get_info(dev)
    budget = int(free * 0.75)
    ex = GpuExecutor(cache)
    # warm-up: a few small requests (kernel attributes, allocator pools)
    rng = np.random.default_rng(100 + rank)
    warm = poisson_requests(rng, max(args.warmup, 3), 1000.0, Nls=spec["nls"], n_range=(1e4, 1e5), maps=(1, 2))
    srv = Server(ex, budget, slots=8).start()
    replay(srv, warm)
    srv.stop(drain=True)
    rng = np.random.default_rng(rank)
    timed = poisson_requests(rng, spec["nreq"], spec["rate"], Nls=spec["nls"], n_range=spec["nrange"],
                             maps=spec["maps"])
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    l0 = lib.dsht_launch_count()
    if world > 1:
        torch.distributed.barrier()
    srv = Server(ex, budget, slots=8).start()
    futs = replay(srv, timed)
    srv.stop(drain=True)
    clk = clocks.stop()
    launches = lib.dsht_launch_count() - l0
    for f in futs:
        f.result()
    st = srv.stats()
    makespan = reduce_scalar(st["makespan_s"], "max", dev)
    pe_all = reduce_scalar(st["points_ell"], "sum", dev)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        value = pe_all / makespan
        line = {"metric": "points*ell/s", "value": value, "unit": "points*ell/s", "n_gpus": world,
                "steps": spec["nreq"], "warmup": len(warm), "ms_per_step": st["mean_ms"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64 NUFFT, i8 tensor-core or f64 direct bin sums (AUTO) + i8 digit-table contraction + f64", "data": "synthetic",
                "config": {"workload": spec["name"], "requests": spec["nreq"], "rate_hz": spec["rate"],
                           "points_ell": st["points_ell"], "budget_GB": budget / 1e9, "slots": 8,
                           "plans_resident_GB": cache.resident_bytes() / 1e9, "parallelism": f"replicas x{world}",
                           "l2": "inputs and tables exceed L2"},
                "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "queue_p50_ms": st["queue_p50_ms"],
                "makespan_s": makespan, "max_concurrent": st["max_concurrent"], "plan_build_s": t_plans,
                "e2e": {"value": value, "unit": "points*ell/s", "h2d_bytes_per_step": None,
                        "d2h_bytes_per_step": None,
                        "path": "every request from host numpy to alm in pinned host memory; a step is a request"},
                "gpu_launches": int(launches), "clocks": clk,
                "note": "ms_per_step is the mean request latency (submit -> alm on host); value over the makespan"}
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--cpu-sample", type=int, default=1_000_000,
                    help="points of the cpu_baseline step (the reference's C transform on the host cores)")
    ap.add_argument("--ref-sample", type=int, default=1_000_000,
                    help="points per step of --impl reference (about 20 s per step on 16 host cores, most of it "
                         "the reference's fixed per-call cost; the line also carries the fixed/per-point split "
                         "and the throughput it implies at the workload's full N)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune-cache", default=None,
                    help="JSON file of the uneven-batch autotuner's choices (default: $DSHT_TUNE_CACHE or "
                         "~/.cache/directsht_b200/autotune.json)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--bin-sums", default="auto", choices=["auto", "nufft", "tc", "fp64"],
                    help="bin sums of the mixed level: type-1 NUFFT, direct tensor-core sums, or the "
                         "library's choice by points per bin key (default)")
    ap.add_argument("--maps-per-pass", type=int, default=0, help="DSHT_TUNE_MAPS_PER_PASS (0: automatic)")
    ap.add_argument("--batch", type=int, default=None,
                    help="point sets per step for the headline (dsht_enqueue_batch); default 8 for c2, else 1")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    spec = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, spec)
    if spec["kind"] == "batch":
        return run_batch(args, spec)
    if spec["kind"] == "serve":
        return run_serve(args, spec)

    import torch
    import torch.distributed as dist
    from directsht_b200 import DirectSHT
    from directsht_b200 import _lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    lib = L.load()
    Nl, Nx, N = spec["Nl"], spec["Nx"], spec["N"]
    maps = spec.get("maps", 1)
    th, ph, w = make_points(spec, seed=rank)
    t0 = time.time()
    d = DirectSHT(Nl, Nx, device=dev)
    t_plan = time.time() - t0
    thd, phd, wd = (torch.from_numpy(a).to(dev) for a in (th, ph, w))
    alm = torch.empty((maps, d.Nlm), dtype=torch.complex128, device=dev)
    nbytes = ct.c_size_t()
    L.check(lib.dsht_workspace_size_maps(d._plan, N, maps, ct.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ct.c_void_p(stream.cuda_stream)
    w_dtype = L.DSHT_W_F32 if w.dtype == np.float32 else L.DSHT_W_F64

    def step(out, t=thd, p=phd, ww=wd):
        if maps == 1 and w_dtype == L.DSHT_W_F64:
            L.check(lib.dsht_execute(d._plan, L.ptr(t), L.ptr(p), L.ptr(ww), N, L.DSHT_MODE_CALL, L.ptr(out),
                                     L.ptr(ws), ws.numel(), sp))
        else:
            L.check(lib.dsht_execute_maps(d._plan, L.ptr(t), L.ptr(p), L.ptr(ww), w_dtype, N, maps, N,
                                          L.DSHT_MODE_CALL, L.ptr(out), L.ptr(ws), ws.numel(), sp))

    def timed(precision, sample_clocks):
        """W warm-up steps, then K timed steps between barriers; per-stage CUDA-event times."""
        d.set_precision(precision)
        for _ in range(args.warmup):
            step(alm)
        L.check(lib.dsht_profile_enable(d._plan, 1))
        stage_ms = (ct.c_double * 5)()
        calls = ct.c_int64()
        L.check(lib.dsht_profile_read(d._plan, stage_ms, ct.byref(calls), 1))
        clocks = ClockSampler(local) if sample_clocks else None
        if clocks:
            clocks.start()
            time.sleep(0.3)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = lib.dsht_launch_count()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        ev[0].record(stream)
        for k in range(args.steps):
            step(alm)
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        launches = lib.dsht_launch_count() - launches0
        clk = clocks.stop() if clocks else None
        per_step = np.array([ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)])
        total_ms = ev[0].elapsed_time(ev[-1])
        L.check(lib.dsht_profile_read(d._plan, stage_ms, ct.byref(calls), 1))
        L.check(lib.dsht_profile_enable(d._plan, 0))
        if world > 1:
            t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        ms_step = total_ms / args.steps
        stages = {n: stage_ms[i] / max(calls.value, 1) for i, n in enumerate(L.STAGES)}
        return {"ms_per_step": ms_step, "value": world * N * maps * Nl / (ms_step / 1e3), "per_step": per_step,
                "stages": stages, "launches": int(launches), "clocks": clk, "alm": alm.clone()}

    if args.maps_per_pass:
        d.tune(maps_per_pass=args.maps_per_pass)
    d.tune(bin_sums=args.bin_sums)
    # the method that runs: AUTO takes the NUFFT from 512 points per bin key on average, the
    # FP64 direct sums below 28 and the tensor-core sums in between (DSHT_TUNE_BIN_SUMS)
    bin_method = args.bin_sums if args.bin_sums != "auto" else (
        "nufft" if N >= 512 * 4 * (Nx - 1) else "fp64" if N < 28 * 4 * (Nx - 1) else "tc")
    # eight point sets per headline step: one contraction pass holds up to eight (32 fold
    # columns), so the table read is shared by all of them
    batch = args.batch if args.batch is not None else (8 if args.workload == "c2" else 1)
    if maps > 1 or w_dtype != L.DSHT_W_F64:
        batch = 1
    single = timed(args.precision, sample_clocks=batch == 1)
    main = single
    if batch > 1:
        # The headline: `batch` independent point sets of the same distribution per step,
        # one dsht_enqueue_batch call (the contraction reads the tables once per three
        # point sets, the rotation shares one recursion); point set 0 is the one above.
        sets = [(thd, phd, wd)] + [tuple(torch.from_numpy(a).to(dev) for a in make_points(spec, seed=1000 * rank + i))
                                   for i in range(1, batch)]
        balm = torch.empty((batch, d.Nlm), dtype=torch.complex128, device=dev)
        bstatus = torch.zeros(batch, dtype=torch.int32, device=dev)
        bnb = ct.c_size_t()
        L.check(lib.dsht_workspace_size_batch(d._plan, N, batch, ct.byref(bnb)))
        bws = torch.empty(bnb.value, dtype=torch.uint8, device=dev)
        vp = lambda xs: (ct.c_void_p * batch)(*[x.data_ptr() for x in xs])
        bth, bph, bw = vp([x[0] for x in sets]), vp([x[1] for x in sets]), vp([x[2] for x in sets])
        balms = vp([balm[i] for i in range(batch)])
        bN = (ct.c_int64 * batch)(*([N] * batch))

        def step_batch():
            L.check(lib.dsht_enqueue_batch(d._plan, batch, bth, bph, bw, bN, L.DSHT_MODE_CALL, balms,
                                           L.ptr(bstatus), L.ptr(bws), bws.numel(), sp))

        for _ in range(args.warmup):
            step_batch()
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.3)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = lib.dsht_launch_count()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        ev[0].record(stream)
        for k in range(args.steps):
            step_batch()
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        launches = lib.dsht_launch_count() - launches0
        clk = clocks.stop()
        for f in bstatus.cpu().numpy():
            L.check(lib.dsht_status(int(f) & 0xffffffff, L.DSHT_MODE_CALL))
        per_step = np.array([ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)])
        total_ms = ev[0].elapsed_time(ev[-1])
        if world > 1:
            t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        ms_b = total_ms / args.steps
        # Stage times of one headline step (untimed, after the timed steps): the library's
        # stage events around every launch of one batched call.
        stage_ms = (ct.c_double * 5)()
        calls = ct.c_int64()
        L.check(lib.dsht_profile_enable(d._plan, 1))
        L.check(lib.dsht_profile_read(d._plan, stage_ms, ct.byref(calls), 1))
        step_batch()
        torch.cuda.synchronize()
        L.check(lib.dsht_profile_read(d._plan, stage_ms, ct.byref(calls), 1))
        L.check(lib.dsht_profile_enable(d._plan, 0))
        bstages = {n: stage_ms[i] for i, n in enumerate(L.STAGES)}
        main = {"ms_per_step": ms_b, "value": world * batch * N * Nl / (ms_b / 1e3), "per_step": per_step,
                "stages": bstages, "launches": int(launches), "clocks": clk, "alm": balm[0:1].clone()}
    other = None
    if args.precision == "mixed" and not args.no_fp64_compare:
        other = timed("fp64", sample_clocks=False)
        d.set_precision(args.precision)
    value, ms_step, per_step, stages = main["value"], main["ms_per_step"], main["per_step"], main["stages"]
    launches, clk = main["launches"], main["clocks"]
    max_rel_err = None
    if other is not None:
        ref = other["alm"]  # (maps, Nlm); error relative to each map's max|alm|
        max_rel_err = float(((main["alm"] - ref).abs().amax(dim=1) / ref.abs().amax(dim=1)).max())

    # Roofline of every stage; the dominant one is reported.
    hbm_peak, bf16_peak, peak_src = measured_peaks()
    C = 8
    while C < (Nl + 15) // 16:
        C *= 2

    f32_tables = args.precision == "mixed"
    # Stage times sum every launch of the step: with several maps, bin sums, fold and rotation
    # ran once per map and the contraction once per pass of maps_per_pass maps.
    # maps per contraction pass: the tensor-core contraction serves up to 8 per table read,
    # the FP64 CUDA-core contraction one
    per_pass = (d.tune()["maps_per_pass"] or (8 if args.precision == "mixed" else 1)) if maps > 1 else 1
    passes = -(-maps // per_pass)
    # point sets per step: the headline step's stage times cover `batch` sets (points, bin
    # sums, fold and rotation once per set; one contraction pass serves all of them)
    nsets = batch

    def stage_roof(name, ms):
        """Roofline of one stage: algorithmic bytes or flops of the whole step (the per-unit
        figures below x the units the step processes) / the stage's measured time."""
        if ms <= 0:
            return None
        if name == "contract":
            eb = 4 if f32_tables else 8
            alg = 2.0 * eb * d.Nlm * Nx * passes
            a = alg / (ms * 1e-3) / 1e9
            kern = ("contract_tc_kernel (tcgen05 kind::i8 on 4-byte digit tables, TMA 3D boxes)" if f32_tables
                    else "contract_stream_kernel (FP64 tables, TMA 2D tiles)")
            return {"kernel": kern, "bound": "hbm", "achieved": a,
                    "peak": hbm_peak, "unit": "GB/s", "frac": a / hbm_peak, "peak_source": peak_src,
                    "algorithmic": f"{2 * eb} B of {'digit' if f32_tables else 'FP64'} table (Yv, Yd) per "
                                   f"(l, m, node) per pass ({passes} passes)"}
        if name == "points":
            alg = 56.0 * N * nsets
            a = alg / (ms * 1e-3) / 1e9
            return {"kernel": "count/scan/scatter (counting sort by bin)", "bound": "hbm", "achieved": a,
                    "peak": hbm_peak, "unit": "GB/s", "frac": a / hbm_peak, "peak_source": peak_src,
                    "algorithmic": "24 B of inputs read + 32 B of sorted record written per point"}
        if name == "bin_sums" and args.precision != "fp64" and bin_method == "nufft":
            # the NUFFT kernel's own FP64 work: per point 132 DFMA of kernel values, 48
            # products and fixed-point conversions of the spread, ~50 for atan2 and the
            # Hermite weights; per piece two complex FFTs of n cells (5 n log2 n each)
            logn = nufft_logn(Nl)
            pieces = nufft_pieces(th, ph, Nx, 0.75, 8192)
            alg = (400.0 * N + pieces * 2 * 5.0 * (1 << logn) * logn * (2 if logn > 12 else 1)) * maps * nsets
            a = alg / (ms * 1e-3) / 1e12
            return {"kernel": "nufft_sums_kernel (FP64 spread, shared-memory FFT)", "bound": "fp64",
                    "achieved": a, "peak": 40.0, "unit": "TFLOP/s", "frac": a / 40.0,
                    "peak_source": "nominal (no measured FP64 figure)",
                    "algorithmic": f"400 flop per point + 10 n log2 n per piece ({pieces} pieces, n = {1 << logn}) "
                                   f"x {nsets} point sets",
                    "bound_note": "the kernel's own limit is its shared-memory pipe (96 32-bit reductions per "
                                  "point for the spread, the in-place FFT): L1/TEX throughput 79 % of peak in the "
                                  "ncu capture summarised in profiles/nufft_sums_c2prof.md; no FP64 peak is "
                                  "measured here, so the fp64 fraction uses the nominal 40 TFLOP/s",
                    "equivalent_direct": {"value": 24.0 * N * Nl * maps * nsets / (ms * 1e-3) / 1e12,
                                          "unit": "TFLOP/s",
                                          "what": "24 flop per (point, m, map) of the direct sums over the "
                                                  "stage time: the rate the direct method would need"}}
        if name == "bin_sums" and args.precision != "fp64" and bin_method == "tc":
            alg = 24.0 * N * Nl * maps * nsets
            a = alg / (ms * 1e-3) / 1e12
            ops = 2.0 * 128 * (2 * C) * 8 * N * maps * nsets
            a_ops = ops / (ms * 1e-3) / 1e12
            return {"kernel": "bin_sums_tc_kernel (tcgen05 kind::i8)", "bound": "tensor", "achieved": a,
                    "peak": bf16_peak, "unit": "TFLOP/s", "frac": a / bf16_peak,
                    "peak_source": f"{peak_src} dense bf16 tensor rate",
                    "algorithmic": "24 flop per (point, m, map): 8 FMA sums + 4 FMA angle step",
                    "int8_slice_ops": {"achieved": a_ops, "peak": 2 * bf16_peak, "unit": "TOP/s",
                                       "frac": a_ops / (2 * bf16_peak),
                                       "what": f"8 int8 slice products of a 128 x {2 * C} x (points) GEMM, "
                                               f"2 op per MAC, against 2 x the bf16 rate (dense int8 on B200)"}}
        if name == "bin_sums":
            alg = 24.0 * N * Nl * maps * nsets
            a = alg / (ms * 1e-3) / 1e12
            return {"kernel": "bin_sums_fp64_kernel", "bound": "fp64", "achieved": a, "peak": 40.0,
                    "unit": "TFLOP/s", "frac": a / 40.0, "peak_source": "nominal (no measured FP64 figure)",
                    "algorithmic": "24 flop per (point, m, map): 8 FMA sums + 4 FMA angle step"}
        if name == "rotate":
            # the products themselves: a real Wigner element d^l_{m m'} (m, m' >= 0, the m' < 0
            # terms folded in by the symmetry of d(pi/2)) times a complex coefficient, 2 FMA per
            # map; the recursion that forms d (shared by the maps of a launch) is not counted
            alg = 2.0 * 2 * sum((l + 1) ** 2 for l in range(Nl)) * maps * nsets
            a = alg / (ms * 1e-3) / 1e12
            return {"kernel": "rotate_back_kernel" if maps * nsets == 1 else "rotate_back_maps_kernel",
                    "bound": "fp64", "achieved": a, "peak": 40.0,
                    "unit": "TFLOP/s", "frac": a / 40.0, "peak_source": "nominal (no measured FP64 figure)",
                    "algorithmic": "2 FMA per (l, m >= 0, m' >= 0, map): real d^l_{mm'}(pi/2) times a complex "
                                   "coefficient (the recursion forming d is not counted)"}
        return None

    roofs = {n: stage_roof(n, ms) for n, ms in stages.items()}
    top = max(stages, key=stages.get)
    roof = dict(roofs[top] or {"kernel": top, "bound": None})
    roof["traffic"] = dram_traffic(top, args.precision + (":tc" if top == "bin_sums" and bin_method == "tc" else ""),
                                   N * nsets, d.Nlm, Nx)
    roof["stage_ms"] = stages[top]

    # End to end from pinned host buffers: inputs copied in and alm copied out every step.
    e2e = None
    if args.e2e_steps > 0 and maps == 1 and w_dtype == L.DSHT_W_F64:
        hp = [torch.from_numpy(a).pin_memory() for a in (th, ph, w)]
        out = torch.empty(2 * d.Nlm, dtype=torch.float64).pin_memory()
        dp = ct.POINTER(ct.c_double)

        def e2e_step():
            L.check(lib.dsht_execute_host(d._plan, ct.cast(hp[0].data_ptr(), dp), ct.cast(hp[1].data_ptr(), dp),
                                          ct.cast(hp[2].data_ptr(), dp), N, L.DSHT_MODE_CALL,
                                          ct.cast(out.data_ptr(), dp)))
        e2e_path = "dsht_execute_host (C ABI, pinned host buffers), wall clock per call"
        h2d = 24 * N
    elif args.e2e_steps > 0:
        hp = [torch.from_numpy(a).pin_memory() for a in (th, ph, w)]
        dbuf = [torch.empty_like(a, device=dev) for a in hp]
        out = torch.empty((maps, d.Nlm), dtype=torch.complex128).pin_memory()

        def e2e_step():
            for h, b in zip(hp, dbuf):
                b.copy_(h, non_blocking=True)
            step(alm, *dbuf)
            out.copy_(alm, non_blocking=True)
            stream.synchronize()
        e2e_path = "pinned host -> device copies, dsht_execute_maps (C ABI), alm -> pinned host; wall clock"
        h2d = sum(a.nbytes for a in (th, ph, w))
    if args.e2e_steps > 0:
        e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / args.e2e_steps
        if world > 1:
            t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": world * N * maps * Nl / e2e_s, "unit": "points*ell/s", "ms_per_step": e2e_s * 1e3,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 16 * d.Nlm * maps, "path": e2e_path}
        # The same transforms back to back through directsht_b200.pipeline.Pipeline: each
        # step still copies its host arrays in and its alm out, but the copies of one step
        # overlap the kernels of the neighbouring steps (two slots in flight).
        from directsht_b200.pipeline import Pipeline
        # three slots: the host collects a result two steps behind, so a slot's next copy-in
        # never waits for the host (with two slots the host's result handling sits in the
        # critical path between one step's kernels and the copy-in of the step after next)
        pipe = Pipeline(d, max_N=N, nmaps=maps, w_dtype=w.dtype, depth=3)
        wmat = torch.from_numpy(np.ascontiguousarray(w if w.ndim == 2 else w[None, :])).pin_memory()
        for _ in range(3):
            pipe.submit(hp[0], hp[1], wmat)
        pipe.drain()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tickets = []
        for k in range(args.e2e_steps):
            tickets.append(pipe.submit(hp[0], hp[1], wmat))
            if len(tickets) > 2:
                pipe.result(tickets.pop(0))
        for tk in tickets:
            pipe.result(tk)
        pipe_s = (time.perf_counter() - t0) / args.e2e_steps
        if world > 1:
            t = torch.tensor([pipe_s], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pipe_s = float(t.item())
        e2e_sync = e2e
        e2e = {"value": world * N * maps * Nl / pipe_s, "unit": "points*ell/s", "ms_per_step": pipe_s * 1e3,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 16 * d.Nlm * maps,
               "path": "directsht_b200.pipeline.Pipeline: pinned host inputs -> device (copy stream), "
                       "dsht_enqueue_maps (C ABI), alm -> pinned host; copies of a step overlap the "
                       "neighbouring steps' kernels (three slots); wall clock over the steps",
               "sync_one_at_a_time": e2e_sync}
        del pipe
        # The host link alone: the same host->device bytes from the same pinned buffers, timed
        # with CUDA events on a copy stream with nothing else running.  Each end-to-end step
        # has to move them, so h2d_bytes / this rate bounds its time from below.
        cps = torch.cuda.Stream(device=dev)
        dsts = [torch.empty_like(a, device=dev) for a in hp[:2]] + [torch.empty_like(wmat, device=dev)]
        srcs = [hp[0], hp[1], wmat]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(cps):
            for _ in range(2):
                for d_, s_ in zip(dsts, srcs):
                    d_.copy_(s_, non_blocking=True)
            e0.record(cps)
            for _ in range(3):
                for d_, s_ in zip(dsts, srcs):
                    d_.copy_(s_, non_blocking=True)
            e1.record(cps)
        cps.synchronize()
        h2d_ms = e0.elapsed_time(e1) / 3
        e2e["h2d_link"] = {"gb_per_s": h2d / (h2d_ms * 1e-3) / 1e9, "ms_per_step": h2d_ms,
                           "what": "pinned host -> device copy of one step's inputs alone (CUDA events, copy "
                                   "stream, nothing else running): the floor of an end-to-end step"}
        del dsts

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_run(spec, args.cpu_sample, 1, 1)
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "error": str(exc)}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {
            "metric": "points*ell/s", "value": value, "unit": "points*ell/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": ("f64" if args.precision != "mixed" else
                      "f64 NUFFT sums + i8 digit-table contraction + f64" if bin_method == "nufft" else
                      "f64 direct sums + i8 digit-table contraction + f64" if bin_method == "fp64" else
                      "i8 tensor sums + i8 digit-table contraction + f64"), "data": "synthetic",
            "config": {"workload": spec["name"], "Nl": Nl, "Nx": Nx, "N": N, "maps": maps,
                       "point_sets_per_step": batch, "precision": args.precision, "bin_sums": bin_method,
                       "l2": f"inputs ({(th.nbytes + ph.nbytes + w.nbytes) / 1e6:.0f} MB) and tables "
                             f"({16 * d.Nlm * Nx / 1e9:.1f} GB FP64) exceed L2 every step",
                       "parallelism": f"replicas x{world}"},
            "p50_ms": float(np.percentile(per_step, 50)), "p99_ms": float(np.percentile(per_step, 99)),
            "stages_ms": stages, "plan_build_s": t_plan, "roofline": roof,
            "stages_note": ("one sort (points) for all maps; bin_sums, fold and rotate summed over all maps "
                            "(bin_sums includes the payload gathers), contract over all passes") if maps > 1 else (
                "stages of one headline step (%d point sets: points, bin_sums, fold and rotate for each, one "
                "contraction pass for all), from the library's stage events in an untimed step after the timed "
                "ones" % batch if batch > 1 else "all stages of one step"),
            "stage_rooflines": {k: v for k, v in roofs.items() if v}, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clk,
        }
        if batch > 1:
            line["mixed_single_transform"] = {"value": single["value"], "ms_per_step": single["ms_per_step"],
                                              "stages_ms": single["stages"],
                                              "p50_ms": float(np.percentile(single["per_step"], 50))}
        if other is not None:
            line["fp64_plain"] = {"value": other["value"], "ms_per_step": other["ms_per_step"],
                                  "stages_ms": other["stages"], "point_sets_per_step": 1}
            line["speedup_vs_fp64_plain"] = value / other["value"]
            line["max_rel_err_vs_fp64"] = max_rel_err
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
