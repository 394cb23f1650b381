#!/usr/bin/env python
"""Benchmark of the B200 pair-histogram hot path: pair-evals/s of the mixed-precision kernel vs the
plain FP64 kernel on the 3D workload (N=65536 points in the unit cube, Float64, L2SF/T2SF/L3SF/T3SF
fused, 64 log bins 1e-4..sqrt(3); seeded synthetic data).

One step = one full pass of the pair loop over the workload (all N(N-1)/2 pairs, every operator).
  value  : mixed kernel, inputs resident in HBM, device outputs; CUDA events on the library's stream,
           L2 flushed (256 MiB write) before every timed step.
  e2e    : the same metric through the C ABI with host buffers: H2D of x,u (pinned) + kernels + D2H of
           sums/counts inside the timed region.
  fp64   : the plain FP64 kernel on the same workload, timed like `value`.
Multi-GPU (--gpus N): one process per GPU (torchrun; `python bench.py --gpus N` launches it itself).
The one workload's upper-triangle tile pairs are cut into N shards of equal pair counts, each rank
runs its shard and one NCCL all-reduce adds the partial histograms inside the timed step (strong
scaling: the whole job's pairs over the slowest rank's time, max over ranks).

--impl reference: the reference's CPU path restated (ThreadedBackend: round-robin outer-index chunks,
per-thread histograms), all host threads, on a bounded sample of the same workload.
"""
import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "structurefunctions.jl_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "pair-evals/s mixed-precision vs FP64 kernel on B200; p50/p99 slice latency"
SP2D_METRIC = "single-pass 2D pair-evals/s (six row updates per pair)"  # the rsp2d lines of both arms

# DRAM bytes per point of one launch of the mixed pair kernel, from ncu captures of the same kernel
# (dram__bytes_read.sum + dram__bytes_write.sum): c1 k_flat1d_mx at N = 16384, 851,200 bytes; c3
# k_joint_mx at N = 32768, 1,255,424 bytes. The read is the packed points once (L2-resident after).
DRAM_BYTES_PER_POINT = {"c1": 851200 / 16384, "c3": 1255424 / 32768}
UNIT = "pair-evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1", choices=["c0", "c1", "c2", "c3", "c4", "r1d", "rjoint", "rsp1d",
                                                       "rsp2d"],
                    help="c0-c4: the benchmark configs; r1d / rjoint / rsp1d / rsp2d: the reference's own published "
                         "GPU shapes (N = 20000; rsp1d / rsp2d the one- and two-dimensional single pass)")
    ap.add_argument("--requests", type=int, default=2000, help="c4: number of requests")
    ap.add_argument("--rate", type=float, default=200.0, help="c4: Poisson arrival rate per second")
    ap.add_argument("--slots", type=int, default=256, help="c4: slices resident at once (admission slots)")
    ap.add_argument("--round-pairs", type=float, default=6e9, help="c4: pair budget of one batched round")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target CPU-baseline sample length")
    ap.add_argument("--profile", type=int, default=0, metavar="N",
                    help="profiling case: run the pair kernels of --config on its first N points (a warm-up "
                         "run then two runs per precision) and exit; sized for ncu captures")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"])
    return ap.parse_args()


def run_profile_case(args):
    """Small, self-contained case for ncu: no timing output, a handful of launches."""
    import torch

    from sfb200 import _abi, _lib, synthetic
    from sfb200.api import plan_description

    w = synthetic.config(args.config, n=args.profile)
    ctx = _lib.Context(0)
    xd = torch.from_numpy(np.ascontiguousarray(w.x.T)).cuda()
    ud = torch.from_numpy(np.ascontiguousarray(w.u.T)).cuda()
    precs = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    for prec in precs:
        desc, keep = plan_description(w.ops, w.u.shape[0], w.distance_bins, w.value_bins, w.metric, prec,
                                      w.x.dtype, w.u.dtype)
        plan = _lib.Plan(ctx, desc, keep)
        sums = torch.zeros(plan.n_sums, dtype=torch.float64, device="cuda")
        counts = torch.zeros(plan.n_counts, dtype=torch.int64, device="cuda")
        flags = _abi.RUN_DEVICE_INPUT | _abi.RUN_DEVICE_OUTPUT
        for _ in range(3):
            plan.run(xd.data_ptr(), ud.data_ptr(), w.n, flags, sums.data_ptr(), counts.data_ptr(), ctx.stream)
        st = plan.stats()
        print(json.dumps({"profile_case": w.name, "precision": prec, "kernel_ms": st["kernel_ms"],
                          "tile": st["tile"], "blocks": st["blocks"], "privatization": st["privatization"]}))
        plan.close()
    ctx.close()


# ------------------------------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [t.strip() for t in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------ ours

def measure_peak(device, fp64):
    lib = C.CDLL(os.path.join(ROOT, "structurefunctions.jl_b200", "libsfb200_probe.so"))
    lib.sfb200_probe_fma.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    t, ms = C.c_double(), C.c_double()
    rc = lib.sfb200_probe_fma(device, 1 if fp64 else 0, C.byref(t), C.byref(ms))
    return t.value if rc == 0 else None


def run_ours(args):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    import sfb200 as SF
    from sfb200 import _abi, _lib, synthetic
    from sfb200.api import plan_description
    from sfb200.distributed import allreduce_histogram, shard_value

    w = synthetic.config(args.config)
    x_host = np.asfortranarray(w.x)
    u_host = np.asfortranarray(w.u)
    n = w.n
    pairs = w.pairs
    ctx = _lib.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))

    # device-resident inputs: column-major (W, N) == row-major (N, W)
    xd = torch.from_numpy(np.ascontiguousarray(x_host.T)).cuda()
    ud = torch.from_numpy(np.ascontiguousarray(u_host.T)).cuda()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def make(precision):
        desc, keep = plan_description(w.ops, w.u.shape[0], w.distance_bins, w.value_bins, w.metric, precision,
                                      w.x.dtype, w.u.dtype)
        plan = _lib.Plan(ctx, desc, keep)
        if dist:  # this rank's shard of the tile pairs; one all-reduce adds the shards
            plan.set_option(_abi.OPT_SHARD, shard_value(rank, world))
        sums = torch.zeros(plan.n_sums, dtype=torch.float64, device="cuda")
        counts = torch.zeros(plan.n_counts, dtype=torch.int64, device="cuda")
        return plan, sums, counts

    def device_steps(plan, sums, counts, steps, warmup):
        flags = _abi.RUN_DEVICE_INPUT | _abi.RUN_DEVICE_OUTPUT
        launches = 0
        kernel_ms = []
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                plan.run(xd.data_ptr(), ud.data_ptr(), n, flags, sums.data_ptr(), counts.data_ptr(), ctx.stream)
                if dist:
                    allreduce_histogram(sums, counts)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        total = 0.0
        with torch.cuda.stream(stream):
            for _ in range(steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                plan.run(xd.data_ptr(), ud.data_ptr(), n, flags, sums.data_ptr(), counts.data_ptr(), ctx.stream)
                if dist:
                    allreduce_histogram(sums, counts)
                e1.record(stream)
                e1.synchronize()
                total += e0.elapsed_time(e1)
                st = plan.stats()
                kernel_ms.append(st["kernel_ms"])
                launches += st["kernel_launches"]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        return total, kernel_ms, launches, plan.stats()

    clocks = ClockSampler(local)
    mixed, msums, mcounts = make("mixed")
    fp64, fsums, fcounts = make("fp64")
    fp32, hsums, hcounts = make("fp32")
    # the sphere's FP64 kernel in the reference's own formulation (the pair frame for every pair); the
    # default FP64 kernel runs the mixed kernel's chord algorithm in FP64 (the like-for-like comparison)
    fp64r = None
    if w.metric.__class__.__name__ != "Euclidean" and w.value_bins is None:
        fp64r, rsums, rcounts = make("fp64")
        fp64r.set_option(_abi.OPT_FORMULATION, 1)

    clocks.start()
    t_mixed, kms_mixed, launches_mixed, st_mixed = device_steps(mixed, msums, mcounts, args.steps, args.warmup)
    t_fp64, kms_fp64, launches_fp64, st_fp64 = device_steps(fp64, fsums, fcounts, args.steps, args.warmup)
    t_fp32, kms_fp32, launches_fp32, st_fp32 = device_steps(fp32, hsums, hcounts, args.steps, args.warmup)
    t_fp64r = kms_fp64r = None
    if fp64r is not None:
        t_fp64r, kms_fp64r, _, _ = device_steps(fp64r, rsums, rcounts, args.steps, args.warmup)
    clk = clocks.stop()

    # counts of the kernels must agree (bit-exact binning in all); sums: per-bin deviation of the
    # mixed and FP32-bulk kernels from the FP64 kernel at the full size (relative to |FP64 sum|)
    same_counts = bool(torch.equal(mcounts, fcounts)) and bool(torch.equal(hcounts, fcounts))
    if fp64r is not None:
        same_counts = same_counts and bool(torch.equal(rcounts, fcounts))

    def max_rel_dev(a, b):
        # per operator: max over bins of |a - b| / |b| (sign-definite operators: the tolerance figure;
        # signed ones: near-cancelling bins make it large, see the CPU-oracle parity tests)
        a = a.cpu().numpy().reshape(-1, mixed.n_counts if w.value_bins is None else mixed.n_sums)
        b = b.cpu().numpy().reshape(a.shape)
        out = []
        for k in range(a.shape[0]):
            ok = np.isfinite(b[k]) & (np.abs(b[k]) > 0)
            out.append(float(np.max(np.abs(a[k][ok] - b[k][ok]) / np.abs(b[k][ok]))) if ok.any() else 0.0)
        return out

    dev_mixed = max_rel_dev(msums, fsums)
    dev_fp32 = max_rel_dev(hsums, fsums)

    # e2e through the C ABI with host buffers (pinned): H2D of x and u, the pair kernel, [the
    # all-reduce of the shards,] D2H of the histogram; timed with CUDA events on the library's stream
    xp = torch.from_numpy(np.ascontiguousarray(x_host.T)).pin_memory()
    up = torch.from_numpy(np.ascontiguousarray(u_host.T)).pin_memory()
    hs = torch.zeros(mixed.n_sums, dtype=torch.float64).pin_memory()
    hc = torch.zeros(mixed.n_counts, dtype=torch.int64).pin_memory()

    def e2e_step():
        if dist:
            mixed.run(xp.data_ptr(), up.data_ptr(), n, _abi.RUN_DEVICE_OUTPUT, msums.data_ptr(), mcounts.data_ptr(),
                      ctx.stream)
            allreduce_histogram(msums, mcounts)
            hs.copy_(msums, non_blocking=True)
            hc.copy_(mcounts, non_blocking=True)
        else:
            mixed.run(xp.data_ptr(), up.data_ptr(), n, 0, hs.data_ptr(), hc.data_ptr(), ctx.stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2e_total = 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            e2e_step()
            e1.record(stream)
            e1.synchronize()
            e2e_total += e0.elapsed_time(e1) * 1e-3
    torch.cuda.synchronize()

    def max_over_ranks(v):
        if not dist:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    t_mixed = max_over_ranks(t_mixed)
    t_fp64 = max_over_ranks(t_fp64)
    e2e_total = max_over_ranks(e2e_total * 1e3)

    t_fp32 = max_over_ranks(t_fp32)
    if fp64r is not None:
        t_fp64r = max_over_ranks(t_fp64r)
    ms_mixed = t_mixed / args.steps
    ms_fp64 = t_fp64 / args.steps
    ms_fp32 = t_fp32 / args.steps
    # one workload, its tile pairs sharded over the ranks: the whole job's pairs over the slowest rank
    value = pairs / (ms_mixed * 1e-3)
    fp64_value = pairs / (ms_fp64 * 1e-3)
    fp32_value = pairs / (ms_fp32 * 1e-3)
    e2e_value = pairs / (e2e_total / args.steps * 1e-3)

    kmed_mixed = sorted(kms_mixed)[len(kms_mixed) // 2]
    kmed_fp64 = sorted(kms_fp64)[len(kms_fp64) // 2]
    kmed_fp32 = sorted(kms_fp32)[len(kms_fp32) // 2]
    peak32 = measure_peak(local, False)
    peak64 = measure_peak(local, True)
    flops = w.flops_per_pair
    # per launch: this rank's share of the pairs
    achieved = flops * (pairs / world) / (kmed_mixed * 1e-3) / 1e12
    achieved64 = flops * (pairs / world) / (kmed_fp64 * 1e-3) / 1e12
    # DRAM bytes of one launch of the mixed kernel: measured with ncu (dram__bytes_read.sum +
    # dram__bytes_write.sum) on a smaller case of the same kernel and scaled by N (the traffic is the
    # compulsory read of the packed points, linear in N, not in pairs)
    traffic = DRAM_BYTES_PER_POINT[args.config] * n if args.config in DRAM_BYTES_PER_POINT else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_mixed,
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "f64+f32",
            "precision": "mixed: FP64 point differences, squared distance (exact bin) and projection numerators; "
                         "FP32 normalisation, operator powers and per-lane run accumulation; FP64 merge",
            "data": "synthetic (seeded; no dataset)",
            "config": {
                "workload": w.name,
                "n_points": n,
                "pairs_per_step": pairs,
                "operators": [repr(o) for o in w.ops],
                "distance_bins": len(w.distance_bins) - 1,
                "l2": "flushed before every timed step (256 MiB write); inputs 3 MB",
                "parallelism": f"tile-pair shards x{world}, one NCCL all-reduce of the histogram" if world > 1 else "single GPU",
                "tile": st_mixed["tile"],
                "blocks": st_mixed["blocks"],
            },
            "fp64": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms_fp64, "kernel_ms": kmed_fp64,
                     "roofline_frac_fp64": (achieved64 / peak64) if peak64 else None,
                     "formulation": "the mixed kernel's algorithm with every step in FP64"},
            "fp32": {"value": fp32_value, "unit": UNIT, "ms_per_step": ms_fp32, "kernel_ms": kmed_fp32,
                     "rechecked_pairs_per_step": st_fp32["rechecked"],
                     "max_rel_dev_vs_fp64_per_operator": dev_fp32,
                     "note": "FP32-bulk kernel: FP32 differences, FP64 recheck of bin membership only"},
            "mixed_over_fp64": value / fp64_value,
            **({"fp64_reference_formulation": {
                "value": pairs / (t_fp64r / args.steps * 1e-3), "unit": UNIT, "ms_per_step": t_fp64r / args.steps,
                "kernel_ms": sorted(kms_fp64r)[len(kms_fp64r) // 2],
                "note": "FP64 kernel in the reference's formulation: the pair frame (geodesic frame, parallel "
                        "transport, atan2) for every pair"},
                "mixed_over_fp64_reference_formulation": value / (pairs / (t_fp64r / args.steps * 1e-3))}
               if fp64r is not None else {}),
            "counts_equal_all_precisions": same_counts,
            "mixed_max_rel_dev_vs_fp64_per_operator": dev_mixed,
            "rechecked_pairs_per_step": st_mixed["rechecked"],
            "roofline": {
                "bound": "fp32",
                "achieved": achieved,
                "peak": peak32,
                "unit": "TFLOP/s",
                "frac": (achieved / peak32) if peak32 else None,
                "traffic": traffic,
                "flops_per_pair": flops,
                "flops_per_pair_source": "reference FP64 formula (frozen in synthetic.FLOPS); the mixed kernel's own "
                                         f"formulation performs {synthetic.KERNEL_FLOPS[args.config]} per pair",
                "kernel_ms": kmed_mixed,
                "peak_source": "measured FP32 FMA probe on this GPU (MEASURED_PEAKS.json has no FP32 vector "
                               "figure); nominal 148 SM x 128 lanes x 2 x clock",
            },
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(x_host.nbytes + u_host.nbytes),
                    "d2h_bytes_per_step": int(mixed.n_sums * 8 + mixed.n_counts * 8 + 8)},
            "gpu_launches": launches_mixed,
            "clocks": clk,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    mixed.close()
    fp64.close()
    fp32.close()
    if fp64r is not None:
        fp64r.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()


# ------------------------------------------------------------------------------------------ CPU

def cpu_sample_rate(w, npts, threads):
    import oracle_py
    from sfb200.api import plan_description

    desc, keep = plan_description(w.ops, w.u.shape[0], w.distance_bins, w.value_bins, w.metric, "fp64",
                                  w.x.dtype, w.u.dtype)
    x = w.x[:, :npts]
    u = w.u[:, :npts]
    t0 = time.perf_counter()
    oracle_py.run(desc, x, u, threads=threads)
    dt = time.perf_counter() - t0
    return npts * (npts - 1) // 2 / dt, dt


def cpu_baseline(w, seconds):
    import oracle_py

    threads = max(1, oracle_py.threads_available())
    rate, _ = cpu_sample_rate(w, min(w.n, 4096), threads)
    npts = int(min(w.n, math.sqrt(2.0 * rate * seconds)))
    rate, dt = cpu_sample_rate(w, npts, threads)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {npts} points of the workload ({npts * (npts - 1) // 2} pairs), {dt:.1f} s; "
                      "C restatement of ThreadedBackend (round-robin outer-index chunks, per-thread histograms)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import oracle_py
    from sfb200 import synthetic

    if args.config == "c4":
        print(json.dumps({"impl": "reference", "unavailable": "no CPU arm for c4: the oracle restates the pair "
                          "loops, not the serving loop"}))
        return
    w = synthetic.config(args.config)
    threads = max(1, oracle_py.threads_available())
    rate0, _ = cpu_sample_rate(w, min(w.n, 4096), threads)
    per_step = 2.0 if args.steps <= 10 else 1.0
    npts = int(min(w.n, math.sqrt(2.0 * rate0 * per_step)))
    for _ in range(args.warmup):
        cpu_sample_rate(w, min(npts, 2048), threads)
    total, pairs = 0.0, 0
    for _ in range(args.steps):
        r, dt = cpu_sample_rate(w, npts, threads)
        total += dt
        pairs += npts * (npts - 1) // 2
    value = pairs / total
    line = {
        "impl": "reference",
        "metric": SP2D_METRIC if args.config == "rsp2d" else METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": w.name, "sample_points_per_step": npts},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"first {npts} of {w.n} points per step; C restatement of the reference "
                                   "ThreadedBackend (no Julia toolchain on this machine)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------ serving

def _percentiles(v, qs=(50, 99)):
    v = np.asarray(v, dtype=np.float64)
    return {f"p{q}": float(np.percentile(v, q)) for q in qs} if v.size else {f"p{q}": None for q in qs}


def run_serving(args):
    """c4: a stream of requests with Poisson arrivals, served by the continuous-batching loop, then
    by one launch per request (FIFO, same arrival times); latencies from arrival to result."""
    import threading

    import torch

    import sfb200 as SF  # noqa: F401
    from sfb200 import _lib, synthetic
    from sfb200.api import plan_description
    from sfb200.serving import GpuExecutor, Request, Server

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and rank != 0:
        return  # the serving run is a single-GPU measurement (requests are not sharded here)
    torch.cuda.set_device(local)
    workers = max(1, min(16, (os.cpu_count() or 2) - 1))
    t_gen = time.perf_counter()
    reqs = synthetic.serving_requests(count=args.requests, rate=args.rate, workers=workers)
    warm = synthetic.serving_requests(count=max(3, args.warmup) * 6, rate=1e9, seed=99, n_max=5000)
    t_gen = time.perf_counter() - t_gen

    def subrequests(q):
        out = [Request(q["ops"], q["x"], q["u"], q["edges"], None, q["metric"])]
        if q["value_bins"] is not None:
            out.append(Request((SF.ProjectedStructureFunctionType(1, 0),), q["x"], q["u"], q["edges"],
                               q["value_bins"], q["metric"]))
        return out

    def pairs_of(q):
        return q["n"] * (q["n"] - 1) // 2 * (2 if q["value_bins"] is not None else 1)

    total_pairs = sum(pairs_of(q) for q in reqs)

    # ---- batched
    ex = GpuExecutor(local)
    clocks = ClockSampler(local)
    srv = Server(ex, max_slots=args.slots, round_pairs=args.round_pairs).start()
    for q in warm:
        for r in subrequests(q):
            srv.submit(r).wait(120)
    rounds0 = srv.rounds
    ex.launches = 0
    tickets = [None] * len(reqs)
    clocks.start()
    t0 = time.perf_counter() + 0.05

    def feeder():
        for k, q in enumerate(reqs):
            d = t0 + q["t"] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[k] = (time.perf_counter(), [srv.submit(r) for r in subrequests(q)])

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    lat_b, done_b = [], []
    for k, (ta, ts) in enumerate(tickets):
        for t in ts:
            t.wait(600)
        done = max(t.t_done for t in ts)
        lat_b.append(done - ta)
        done_b.append(done)
    clk = clocks.stop()
    srv.stop()
    rounds = srv.rounds - rounds0
    launches = ex.launches
    span_b = max(done_b) - t0
    ex.close()

    # ---- one launch per request (FIFO on the same arrivals), each request's service time alone
    ctx = _lib.Context(local)
    plans = {}

    def plan_for(r):
        key = (tuple(repr(o) for o in r.ops), r.u.shape[0], repr(r.metric), r.x.dtype.str, r.u.dtype.str,
               np.asarray(r.distance_bins).tobytes(), repr(r.value_bins))
        if key not in plans:
            desc, keep = plan_description(r.ops, r.u.shape[0], r.distance_bins, r.value_bins, r.metric, "mixed",
                                          r.x.dtype, r.u.dtype)
            plans[key] = (_lib.Plan(ctx, desc, keep), keep)
        return plans[key][0]

    def run_alone(r):
        p = plan_for(r)
        s = np.zeros(p.n_sums)
        c = np.zeros(p.n_counts, dtype=np.uint64)
        xa, ua = np.asfortranarray(r.x), np.asfortranarray(r.u)
        p.run(xa.ctypes.data, ua.ctypes.data, r.n, 0, s.ctypes.data, c.ctypes.data)

    for q in warm:
        for r in subrequests(q):
            run_alone(r)
    subs = [subrequests(q) for q in reqs]
    t0 = time.perf_counter() + 0.05
    lat_1, svc_1, done_1 = [], [], []
    for q, rs in zip(reqs, subs):
        ta = t0 + q["t"]
        d = ta - time.perf_counter()
        if d > 0:
            time.sleep(d)
        ts = time.perf_counter()
        for r in rs:
            run_alone(r)
        te = time.perf_counter()
        lat_1.append(te - ta)
        svc_1.append(te - ts)
        done_1.append(te)
    span_1 = max(done_1) - t0
    for p, _ in plans.values():
        p.close()
    ctx.close()

    lat_b = np.array(lat_b)
    lat_1 = np.array(lat_1)
    svc = np.array(svc_1)
    slow_b = lat_b / svc
    slow_1 = lat_1 / svc
    sizes = np.array([pairs_of(q) for q in reqs], dtype=np.float64)
    deciles = []
    edges = np.quantile(sizes, np.linspace(0, 1, 11))
    for k in range(10):
        m = (sizes >= edges[k]) & ((sizes <= edges[k + 1]) if k == 9 else (sizes < edges[k + 1]))
        deciles.append({"pairs": [float(edges[k]), float(edges[k + 1])], "n": int(m.sum()),
                        "latency_ms": {kk: v * 1e3 for kk, v in _percentiles(lat_b[m]).items()},
                        "slowdown": _percentiles(slow_b[m])})
    value = total_pairs / span_b
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": 1,
        "steps": len(reqs),
        "warmup": len(warm),
        "ms_per_step": float(np.mean(lat_b) * 1e3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64+f32",
        "data": "synthetic (seeded; no dataset)",
        "config": {"workload": f"c4 serving: {len(reqs)} requests, Poisson {args.rate}/s, N log-uniform "
                               "[1e3, 1e5], 2D/3D planar or spherical, 32-64 log bins, order 2 or 3, half with "
                               "the 256-value-bin joint histogram",
                   "total_pairs": int(total_pairs), "step": "one request (1D and, if asked, joint histogram)",
                   "l2": "inputs of a request are copied from host memory at admission (no flush needed)",
                   "max_slots": args.slots, "round_pairs": args.round_pairs, "generation_s": t_gen},
        "latency": {"raw_ms": {k: v * 1e3 for k, v in _percentiles(lat_b).items()},
                    "slowdown": _percentiles(slow_b),
                    "slowdown_p99_over_p50": float(np.percentile(slow_b, 99) / np.percentile(slow_b, 50)),
                    "raw_p99_over_p50": float(np.percentile(lat_b, 99) / np.percentile(lat_b, 50)),
                    "by_size_decile": deciles,
                    "slowdown_definition": "latency / the request's service time when run alone (one launch "
                                           "per histogram, measured in the baseline run)"},
        "rounds": rounds,
        "one_launch_per_request": {"value": total_pairs / span_1, "unit": UNIT,
                                   "latency_raw_ms": {k: v * 1e3 for k, v in _percentiles(lat_1).items()},
                                   "slowdown": _percentiles(slow_1)},
        "batched_over_one_launch": (total_pairs / span_b) / (total_pairs / span_1),
        "e2e": {"value": value, "unit": UNIT,
                "h2d_bytes_per_step": int(np.mean([q["x"].nbytes + q["u"].nbytes for q in reqs])),
                "d2h_bytes_per_step": int(np.mean([8 * 2 * (len(q["edges"]) - 1) *
                                                   (1 + (256 if q["value_bins"] is not None else 0))
                                                   for q in reqs]))},
        "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_single_pass_2d(args):
    """rsp2d: the two-dimensional single pass of one point set, as the public call runs it -- the rows
    (S2, L2, T2, S3, L3, L1T2) grouped into as few joint launches as their cells allow (one for the six
    rows here, sfb200.single_pass._rows_per_launch) on the device-resident points, the launches of a
    step timed together with CUDA events on the library's stream, L2 flushed between steps. The metric
    counts each pair once (its six row updates included), as the reference's SP2D rate does. Runs on
    rank 0 only (one point set; the other ranks exit without work)."""
    import torch

    if int(os.environ.get("RANK", "0")) != 0:
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from sfb200 import _abi, _lib, synthetic
    from sfb200.api import plan_description
    from sfb200.single_pass import SINGLE_PASS_N, _rows_per_launch

    w = synthetic.config("rsp2d")
    nd, nv = len(w.distance_bins) - 1, len(w.value_bins) - 1
    k_rows = _rows_per_launch([w.value_bins] * SINGLE_PASS_N, nd, nv, w.metric, 2)
    groups = [w.ops[t:t + k_rows] for t in range(0, SINGLE_PASS_N, k_rows)]
    ctx = _lib.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    xd = torch.from_numpy(np.ascontiguousarray(np.asfortranarray(w.x).T)).cuda()
    ud = torch.from_numpy(np.ascontiguousarray(np.asfortranarray(w.u).T)).cuda()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    flags = _abi.RUN_DEVICE_INPUT | _abi.RUN_DEVICE_OUTPUT
    precisions = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    clocks = ClockSampler(local)
    out, counts_of = {}, {}
    # the precisions on the grouped launches, then FP64 with one launch per row (the form before grouping)
    variants = [(prec, prec, groups) for prec in precisions] + [("fp64, one launch per row", "fp64",
                                                                 [(op,) for op in w.ops])]
    for k, (label, prec, vgroups) in enumerate(variants):
        rows = []
        for ops in vgroups:
            desc, keep = plan_description(ops, 2, w.distance_bins, w.value_bins, w.metric, prec, w.x.dtype, w.u.dtype)
            plan = _lib.Plan(ctx, desc, keep)
            rows.append((plan, torch.zeros(plan.n_sums, dtype=torch.float64, device="cuda"),
                         torch.zeros(plan.n_counts, dtype=torch.int64, device="cuda")))

        def step():
            for plan, sums, counts in rows:
                plan.run(xd.data_ptr(), ud.data_ptr(), w.n, flags, sums.data_ptr(), counts.data_ptr(), ctx.stream)

        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                step()
        torch.cuda.synchronize()
        if k == 0:
            clocks.start()
        total, kernel_ms, launches = 0.0, [], 0
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step()
                e1.record(stream)
                e1.synchronize()
                total += e0.elapsed_time(e1)
                sts = [plan.stats() for plan, _, _ in rows]
                kernel_ms.append([st["kernel_ms"] for st in sts])
                launches += sum(st["kernel_launches"] for st in sts)
        torch.cuda.synchronize()
        ms = total / args.steps
        out[label] = {"value": w.pairs / (ms * 1e-3), "ms_per_step": ms, "gpu_launches": launches,
                      "rows_per_launch": len(vgroups[0]),
                      "launch_kernel_ms": [round(min(r[t] for r in kernel_ms), 4) for t in range(len(rows))],
                      "rechecked": [st["rechecked"] for st in sts]}
        counts_of[label] = np.concatenate([c.cpu().numpy() for _, _, c in rows])
        for plan, _, _ in rows:
            plan.close()
    clk = clocks.stop()
    head = out[precisions[0]]
    line = {"metric": SP2D_METRIC, "value": head["value"],
            "unit": "pair-evals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "replicas only",
            "vs_baseline": None, "dtype": "f64",  # flat single-pass 2D rows run the FP64 joint kernel at either precision
            "data": "synthetic (seeded; no dataset)",
            "config": {"workload": w.name, "precision": precisions[0], "l2": "flushed between steps"},
            "gpu_launches": head["gpu_launches"], "clocks": clk,
            "reference_published": {"value": 2.8e10, "unit": "pair-evals/s", "hardware": "A100",
                                    "source": "gpu/OPTIMAL_KERNEL_DESIGN.md:186,210-216 (64 slices of 20000 points)"},
            "variants": out}
    first = next(iter(counts_of.values()))
    line["counts_equal"] = all(np.array_equal(first, c) for c in counts_of.values())
    if not args.no_cpu_baseline:  # the oracle's six-row pass (the reference's own loop) on the host cores
        line["cpu_baseline"] = cpu_baseline(w, args.cpu_seconds)
    print(json.dumps(line), flush=True)
    ctx.close()


def spawn_ranks(n):
    """`--gpus N` without a launcher: run this script as N ranks under torch.distributed.run (one
    process per GPU, rendezvous on 127.0.0.1) and return its exit status."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd, cwd=ROOT)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    if args.warmup < 3:
        args.warmup = 3
    if args.profile:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config == "c4":
        run_serving(args)
    elif args.config == "rsp2d":
        run_single_pass_2d(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
