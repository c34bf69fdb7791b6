#!/usr/bin/env python
"""Benchmark of the strack hot path on the large synthetic pair.

Workload: 12000 az x 24000 rg complex64 pair (coherence per 512-px block in
[0.3, 0.9], displacement up to 12 px), complex window 64 x 64 with amplitude
fallback, grid step 24 rg x 6 az: 1969 x 993 = 1,955,217 patches per step.
A step is one full sb_strack call over that grid.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

value : patches/s with both images already resident in HBM (device time of
        the whole call, CUDA events on the library's stream);
e2e   : patches/s through the C ABI with big-endian host images in pinned
        memory; every step copies both images host->device and the five
        output grids device->host inside the timed region.
Inputs (4.6 GB) are far larger than L2 (126 MB), so no flush is needed.
accuracy: the last step's offsets against the FP64 oracle on a spread sample
        of grid rows (one per host core): error percentiles in px, the
        fraction within 0.02 px (0.01 px for complex matches), match agreement.
Under torchrun every rank tracks its own pair (weak scaling, no collective on
the data path); rank 0 prints the max-over-ranks time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NA, NR = 12000, 24000
W = 64
GRID = dict(rStart=96, aStart=96, deltaR=24, deltaA=6, wR=W, wA=W, wRa=W, wAa=W)
N_R = (NR - 2 * GRID["rStart"]) // GRID["deltaR"] + 1  # 993
N_A = (NA - 2 * GRID["aStart"]) // GRID["deltaA"] + 1  # 1969


METRIC = "patches/s at <=0.02 px err vs FP64 oracle (plain FP32); p50/p99 ms"


def use_small_workload():
    """2400 x 4800 pair of the same generator (71,217 patches): the profiling case."""
    global NA, NR, N_R, N_A
    NA, NR = 2400, 4800
    N_R = (NR - 2 * GRID["rStart"]) // GRID["deltaR"] + 1
    N_A = (NA - 2 * GRID["aStart"]) // GRID["deltaA"] + 1


def _alg_flops_fft(n_points):
    import math
    return 5.0 * n_points * math.log2(n_points)


# algorithmic work per point (FFT flop count of the reference's transforms)
ALG_CMPLX = 2 * _alg_flops_fft(W * W) + _alg_flops_fft(4 * W * W) + _alg_flops_fft(64) + _alg_flops_fft(96 * 96) \
    + 6 * W * W
ALG_AMP_S = 2 * _alg_flops_fft(W * W) + 5 * _alg_flops_fft(4 * W * W) + _alg_flops_fft(64) \
    + _alg_flops_fft(96 * 96)
ALG_AMP_L = 2 * _alg_flops_fft(4 * W * W) + 5 * _alg_flops_fft(16 * W * W) + _alg_flops_fft(64) \
    + _alg_flops_fft(96 * 96)


def track_params():
    from specklesource_b200 import abi
    return abi.TrackParams(nR=N_R, nA=N_A, **GRID)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm_load = [s for s in sm if smax and s > 0.3 * smax] or sm
        return {"sm_mhz": float(np.median(sm_load)) if sm_load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp32_peak_tflops(torch):
    """FP32 CUDA-core reference: cuBLAS SGEMM (TF32 off), best of 5."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda")
    b = torch.randn(n, n, device="cuda")
    best = 0.0
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.mm(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return best


# ---------------------------------------------------------------- CPU baseline

def _cpu_worker(args):
    band1, band2, aStart, nA, precision = args
    sys.path.insert(0, ROOT)
    from oracle import oracle
    from specklesource_b200 import abi
    p = abi.TrackParams(nR=N_R, nA=nA, **dict(GRID, aStart=aStart))
    t = time.time()
    o = oracle.strack(p, band1, band2, precision=precision)
    return time.time() - t, nA * N_R, {k: o[k] for k in ("offR", "offA", "type")}


def _row_jobs(img1, img2, rows_per_worker, workers, precision):
    """One job per worker: rows_per_worker consecutive grid rows, the workers'
    row blocks spread evenly over the grid, each with the image band covering
    every window of its rows (large amplitude window and the secondary image's
    shift included)."""
    jobs, starts = [], []
    for w in range(workers):
        i0 = min(N_A - rows_per_worker, (w * N_A) // workers)
        a_lo = GRID["aStart"] + i0 * GRID["deltaA"] - W - 32
        a_hi = GRID["aStart"] + (i0 + rows_per_worker - 1) * GRID["deltaA"] + 2 * W + 32
        lo = max(0, a_lo)
        b1 = np.ascontiguousarray(img1[lo:a_hi])
        b2 = np.ascontiguousarray(img2[lo:a_hi])
        # aStart relative to the band keeps the window coordinates of the full grid
        jobs.append((b1, b2, GRID["aStart"] + i0 * GRID["deltaA"] - lo, rows_per_worker, precision))
        starts.append(i0)
    return jobs, starts


def _run_pool(jobs):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(len(jobs)) as pool:
        res = pool.map(_cpu_worker, jobs)
    return res, time.time() - t0


def cpu_baseline(img1, img2, rows_per_worker=6, workers=None):
    """The f32 oracle (reference-like precision) on rows_per_worker grid rows per
    process, all host cores, spawned processes over azimuth bands spread over
    the grid."""
    workers = workers or os.cpu_count()
    jobs, _ = _row_jobs(img1, img2, rows_per_worker, workers, "f32")
    res, wall = _run_pool(jobs)
    pts = sum(r[1] for r in res)
    work = max(r[0] for r in res)
    return {"value": pts / work, "unit": "patches/s", "cores": workers, "kind": "port",
            "sample": f"{workers} processes x {rows_per_worker} grid rows x {N_R} patches ({pts} patches) of "
                      f"the same workload spread over the grid, f32 CPU restatement (oracle/, gcc -O3), "
                      f"{work:.1f} s compute, {wall:.1f} s wall incl. spawn"}


def accuracy_vs_fp64(img1, img2, gpu, rows_per_worker=1, workers=None):
    """Offsets of the GPU run against the FP64 oracle on a spread sample of grid
    rows: error percentiles (px) on the points both match, the fraction within
    0.02 px (0.01 px for complex matches), and match-type agreement."""
    workers = workers or os.cpu_count()
    jobs, starts = _row_jobs(img1, img2, rows_per_worker, workers, "f64")
    res, wall = _run_pool(jobs)
    errs, tol_ok, n_match, same, n_pts = [], 0, 0, 0, 0
    for (_, _, o), i0 in zip(res, starts):
        sl = slice(i0, i0 + rows_per_worker)
        g = {k: gpu[k][sl] for k in ("offR", "offA", "type")}
        matched = o["type"] > 0
        both = matched & (g["type"] > 0)
        e = np.maximum(np.abs(g["offR"].astype(np.float64) - o["offR"]),
                       np.abs(g["offA"].astype(np.float64) - o["offA"]))
        tol = np.where(o["type"] == 1, 0.01, 0.02)
        tol_ok += int((both & (e <= tol)).sum())
        n_match += int(matched.sum())
        same += int((g["type"] == o["type"]).sum())
        n_pts += o["type"].size
        errs.append(e[both])
    e = np.concatenate(errs) if errs else np.zeros(0)
    return {"points": n_pts, "oracle_matches": n_match,
            "frac_within_tol": tol_ok / max(1, n_match), "frac_same_type": same / max(1, n_pts),
            "err_px_p50": float(np.percentile(e, 50)) if e.size else None,
            "err_px_p99": float(np.percentile(e, 99)) if e.size else None,
            "err_px_max": float(e.max()) if e.size else None,
            "sample": f"{workers} x {rows_per_worker} grid rows spread over the grid, FP64 oracle, {wall:.1f} s"}


def measured_traffic(kernel_key):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (a 'traffic_bytes_per_launch:' line), or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel_key}.md")
    try:
        with open(path) as f:
            for ln in f:
                if ln.startswith("traffic_bytes_per_launch:"):
                    return int(ln.split(":")[1].strip())
    except (OSError, ValueError):
        return None
    return None


# ---------------------------------------------------------------- main

def pinned_big_endian(torch, t):
    """complex64 CUDA tensor -> big-endian bytes in pinned host memory (numpy '>c8')."""
    na, nr = t.shape
    host = torch.empty((na, nr * 8), dtype=torch.uint8, pin_memory=True)
    rows = max(1, (1 << 28) // (nr * 8))
    for r0 in range(0, na, rows):
        r1 = min(na, r0 + rows)
        b = t[r0:r1].contiguous().view(torch.uint8).reshape(r1 - r0, nr * 2, 4).flip(-1).reshape(r1 - r0, nr * 8)
        host[r0:r1].copy_(b)
    return host.numpy().view(">c8").reshape(na, nr)


def run_reference(args):
    import torch
    from specklesource_b200 import synth
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    s1, s2 = synth.large_pair(device=dev, na=NA, nr=NR)
    a = synth.to_numpy(s1)
    b = synth.to_numpy(s2)
    del s1, s2
    vals = []
    cb = None
    for k in range(args.warmup + args.steps):
        rows = 1 if k < args.warmup else args.cpu_rows
        r = cpu_baseline(a, b, rows_per_worker=rows)
        if k >= args.warmup:
            vals.append(r["value"])
            cb = r
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v,
            "unit": "patches/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * N_A * N_R / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded speckle pair, no public dataset)",
            "config": {"workload": "strack 12000x24000 w64 step 24x6 (1,955,217 patches)",
                       "sample": "bounded CPU sample per step"},
            "cpu_baseline": dict(cb, value=v),
            "e2e": {"value": v, "unit": "patches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-rows", type=int, default=6, help="grid rows per CPU process in the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32-peak", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP64-oracle check of a row sample")
    ap.add_argument("--workload", default="large", choices=["large", "small"],
                    help="small: 2400x4800 profiling case of the same generator")
    args = ap.parse_args()
    if args.workload == "small":
        use_small_workload()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from specklesource_b200 import runtime, synth

    ctx = runtime.Context(local)
    p = track_params()
    s1, s2 = synth.large_pair(device="cuda", na=NA, nr=NR, seed=2 + 7 * rank)
    torch.cuda.synchronize()
    out = {k: torch.empty((N_A, N_R), dtype=torch.float32, device="cuda") for k in ("offR", "offA", "corr", "azd")}
    out["type"] = torch.empty((N_A, N_R), dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    def step_dev():
        ctx.strack(p, s1, s2, out=out)
        return ctx.timing()["total"], ctx.stage_timing(), ctx.launch_count()

    for _ in range(args.warmup):
        step_dev()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    tot_ms, stages, launches, step_ms = 0.0, [], 0, []
    for _ in range(args.steps):
        t, st, nl = step_dev()
        tot_ms += t
        step_ms.append(t)
        stages.append(st)
        launches += nl
    barrier()
    clk = clocks.stop()
    n_pts = N_A * N_R
    ms_step = tot_ms / args.steps
    if world > 1:
        tt = torch.tensor([ms_step], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms_step = float(tt.item())
    value = world * n_pts / (ms_step * 1e-3)

    # ---- roofline of the dominant kernel (complex stage, FP32 CUDA cores)
    st0 = stages[-1]
    cm_ms = float(np.mean([s["cmplx_ms"] for s in stages]))
    ach_tflops = st0["n_cmplx"] * ALG_CMPLX / (cm_ms * 1e-3) / 1e12
    fp32 = float("nan") if args.no_fp32_peak else fp32_peak_tflops(torch)
    peaks, src = measured_peaks()
    img_bytes = 2 * NA * NR * 8

    # ---- end to end through the C ABI with pinned big-endian host images
    e2e = None
    if not args.no_e2e:
        h1 = pinned_big_endian(torch, s1)
        h2 = pinned_big_endian(torch, s2)
        hout = {k: torch.empty((N_A, N_R), dtype=torch.float32, pin_memory=True).numpy()
                for k in ("offR", "offA", "corr", "azd")}
        hout["type"] = torch.empty((N_A, N_R), dtype=torch.uint8, pin_memory=True).numpy()
        for _ in range(max(1, args.warmup)):
            ctx.strack(p, h1, h2, out=hout)
        barrier()
        e_ms = 0.0
        for _ in range(args.steps):
            ctx.strack(p, h1, h2, out=hout)
            e_ms += ctx.timing()["total"]
        barrier()
        e_ms /= args.steps
        if world > 1:
            tt = torch.tensor([e_ms], device="cuda")
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            e_ms = float(tt.item())
        e2e = {"value": world * n_pts / (e_ms * 1e-3), "unit": "patches/s", "h2d_bytes_per_step": img_bytes,
               "d2h_bytes_per_step": n_pts * (4 * 4 + 1), "ms_per_step": e_ms,
               "match_fraction": float((hout["type"] > 0).mean())}

    cpu, acc = None, None
    if rank == 0 and world == 1 and not (args.no_cpu_baseline and args.no_accuracy):
        a = synth.to_numpy(s1)
        b = synth.to_numpy(s2)
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(a, b, rows_per_worker=args.cpu_rows)
        if not args.no_accuracy:
            g = {k: out[k].cpu().numpy() for k in ("offR", "offA", "type")}
            acc = accuracy_vs_fp64(a, b, g)
    key = f"strack_cmplx_w64_{NA}x{NR}"
    traffic = measured_traffic(key)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value, "unit": "patches/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded speckle pair, no public dataset)",
            "config": {"workload": f"strack {NA}x{NR} w64 step 24x6 ({n_pts:,} patches, complex + amplitude "
                                   "fallback)", "parallelism": f"replicas x{world}",
                       "l2": "inputs 4.6 GB >> 126 MB L2, no flush"},
            "e2e": e2e,
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                           "what": "one sb_strack call over the whole grid, images resident"},
            "accuracy": acc,
            "gpu_launches": launches,
            "stages": {k: float(np.mean([s[k] for s in stages])) for k in stages[-1]},
            "roofline": {
                "bound": "fp32", "achieved": ach_tflops, "peak": fp32, "unit": "TFLOP/s",
                "frac": ach_tflops / fp32,
                "traffic": traffic,
                "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, profiles/{key}.md"
                                  if traffic else "no committed capture for this workload",
                "alg_bytes_per_launch": img_bytes + n_pts * (4 * 4 + 1),
                "kernel": "strack_cmplx_kernel<64,512>",
                "alg_flops_per_patch": ALG_CMPLX,
                "peak_source": "cuBLAS SGEMM 8192^3 (TF32 off) measured in this run",
                "hbm": {"achieved_gbs": (img_bytes) / (cm_ms * 1e-3) / 1e9, "peak_gbs": peaks.get("hbm_gbs"),
                        "peak_source": src},
            },
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
