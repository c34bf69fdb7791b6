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
        fraction within 0.02 px (0.01 px for complex matches), match
        agreement, and the per-peak-value (corr) error percentiles.
parity_other_configs: the same figures for cfg1 (whole 1024 x 2048 grid,
        W = 32) and for strackw at the cfg3 geometry (240 points).
Under torchrun every rank tracks its own pair (weak scaling, no collective on
the data path); rank 0 prints the max-over-ranks time.
"""
import argparse
import collections
import dataclasses
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


METRIC = "patches/s at <=0.02 px err vs FP64 oracle (plain FP32 vs split-BF16); p50/p99 ms"


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


def replica_seed(rank):
    """Seed of the synthetic pair rank `rank` tracks (each replica its own pair)."""
    return 2 + 7 * rank


def max_over_ranks(torch, value, world, device):
    """The slowest rank's value: all-reduce MAX over the process group (the
    job's time is set by its slowest replica).  world <= 1: value itself."""
    if world <= 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, n_units, ms):
    """Whole-job units/s of a replica run: every rank processed n_units, the
    slowest in ms milliseconds."""
    return world * n_units / (ms * 1e-3)


# the library runs the complex stage in list chunks of this many patches
# (one complex + one peak launch each; kPeakChunk in csrc/capi.cu)
PEAK_CHUNK = 1 << 19


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
    band1, band2, aStart, nA, nR, precision = args
    sys.path.insert(0, ROOT)
    from oracle import oracle
    from specklesource_b200 import abi
    p = abi.TrackParams(nR=nR, nA=nA, **dict(GRID, aStart=aStart))
    t = time.time()
    o = oracle.strack(p, band1, band2, precision=precision)
    return time.time() - t, nA * nR, {k: o[k] for k in ("offR", "offA", "corr", "type")}


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
        # aStart relative to the band keeps the window coordinates of the full grid;
        # the grid width travels with the job (spawned workers see the default workload)
        jobs.append((b1, b2, GRID["aStart"] + i0 * GRID["deltaA"] - lo, rows_per_worker, N_R, precision))
        starts.append(i0)
    return jobs, starts


def _run_pool(jobs):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(len(jobs)) as pool:
        res = pool.map(_cpu_worker, jobs)
    return res, time.time() - t0


def fft_vs_scipy(sizes=((8, 8), (64, 64), (96, 96), (128, 128))):
    """The CPU baseline's FFT (the f32 oracle's, one thread, plan reused)
    against scipy.fft (pocketfft, one thread) on the transform sizes of the
    default workload: us per 2-D transform and the ratio, so the baseline is
    shown to use a competitive FFT (the reference calls FFTW)."""
    try:
        import scipy.fft
    except ImportError:
        return None
    from oracle import oracle
    out = {}
    rng = np.random.default_rng(0)
    for na, nr in sizes:
        reps = max(5, int(4e6 // (na * nr)))
        to = oracle.fft2d_time(na, nr, reps, "f32")
        x = (rng.standard_normal((na, nr)) + 1j * rng.standard_normal((na, nr))).astype(np.complex64)
        scipy.fft.fft2(x, workers=1)
        t0 = time.perf_counter()
        for _ in range(reps):
            scipy.fft.fft2(x, workers=1)
        ts = (time.perf_counter() - t0) / reps
        out[f"{na}x{nr}"] = {"oracle_us": to * 1e6, "scipy_us": ts * 1e6, "ratio": to / ts}
    return out


def cpu_baseline(img1, img2, rows_per_worker=32, workers=None):
    """The f32 oracle (reference-like precision) on rows_per_worker grid rows per
    process, all host cores, spawned processes over azimuth bands spread over
    the grid."""
    workers = workers or os.cpu_count()
    jobs, _ = _row_jobs(img1, img2, rows_per_worker, workers, "f32")
    res, wall = _run_pool(jobs)
    pts = sum(r[1] for r in res)
    work = max(r[0] for r in res)
    return {"value": pts / work, "unit": "patches/s", "cores": workers, "kind": "port",
            "sample_patches": pts, "sample_s": work,
            "sample": f"{workers} processes x {rows_per_worker} grid rows x {N_R} patches ({pts} patches) of "
                      f"the same workload spread over the grid, f32 CPU restatement (oracle/, gcc -O3, "
                      f"vectorised 2-D FFT), {work:.1f} s compute, {wall:.1f} s wall incl. spawn",
            "fft_vs_scipy": fft_vs_scipy()}


def corr_errors(g_corr, o_corr, both):
    """Per-peak-value error of the GPU's correlation against the FP64 oracle
    on the points both match: absolute and relative percentiles."""
    if not both.any():
        return {"corr_abs_p50": None, "corr_abs_p99": None, "corr_abs_max": None, "corr_rel_p99": None}
    d = np.abs(g_corr[both].astype(np.float64) - o_corr[both])
    r = d / np.maximum(1e-6, np.abs(o_corr[both]))
    return {"corr_abs_p50": float(np.percentile(d, 50)), "corr_abs_p99": float(np.percentile(d, 99)),
            "corr_abs_max": float(d.max()), "corr_rel_p50": float(np.percentile(r, 50)),
            "corr_rel_p99": float(np.percentile(r, 99)), "corr_rel_max": float(r.max())}


def _accuracy_blocks(pairs):
    """Parity figures over (gpu, oracle) grid pieces: offset error percentiles
    (px) and per-peak-value (corr) error on the points both match, the
    fraction within 0.02 px (0.01 px for complex matches), match agreement."""
    errs, gc, oc, ok, n_match, same, n_pts = [], [], [], 0, 0, 0, 0
    for g, o in pairs:
        matched = o["type"] > 0
        both = matched & (g["type"] > 0)
        e = np.maximum(np.abs(g["offR"].astype(np.float64) - o["offR"]),
                       np.abs(g["offA"].astype(np.float64) - o["offA"]))
        tol = np.where(o["type"] == 1, 0.01, 0.02)
        ok += int((both & (e <= tol)).sum())
        n_match += int(matched.sum())
        same += int((g["type"] == o["type"]).sum())
        n_pts += o["type"].size
        errs.append(e[both])
        gc.append(g["corr"][both])
        oc.append(o["corr"][both])
    e = np.concatenate(errs) if errs else np.zeros(0)
    pct = (lambda q: float(np.percentile(e, q)) if e.size else None)
    gcv = np.concatenate(gc) if gc else np.zeros(0, np.float32)
    ocv = np.concatenate(oc) if oc else np.zeros(0)
    out = {"points": n_pts, "oracle_matches": n_match, "frac_within_tol": ok / max(1, n_match),
           "frac_same_type": same / max(1, n_pts), "err_px_p50": pct(50), "err_px_p99": pct(99),
           "err_px_max": float(e.max()) if e.size else None}
    out.update(corr_errors(gcv, ocv, np.ones(gcv.size, bool)))
    return out


def accuracy_vs_fp64(img1, img2, gpu, rows_per_worker=1, workers=None):
    """Offsets and correlations of the GPU run against the FP64 oracle on a
    spread sample of grid rows (see _accuracy_blocks)."""
    workers = workers or os.cpu_count()
    jobs, starts = _row_jobs(img1, img2, rows_per_worker, workers, "f64")
    res, wall = _run_pool(jobs)
    pairs = []
    for (_, _, o), i0 in zip(res, starts):
        sl = slice(i0, i0 + rows_per_worker)
        pairs.append(({k: gpu[k][sl] for k in ("offR", "offA", "corr", "type")}, o))
    out = _accuracy_blocks(pairs)
    out["sample"] = f"{workers} x {rows_per_worker} grid rows spread over the grid, FP64 oracle, {wall:.1f} s"
    return out


def accuracy_vs_fp64_forms(img1, img2, gpu_by_form, rows_per_worker=1, workers=None):
    """accuracy_vs_fp64 for several GPU outputs of the same workload (one per
    transform form) against one FP64 oracle run."""
    workers = workers or os.cpu_count()
    jobs, starts = _row_jobs(img1, img2, rows_per_worker, workers, "f64")
    res, wall = _run_pool(jobs)
    out = {}
    for name, gpu in gpu_by_form.items():
        pairs = []
        for (_, _, o), i0 in zip(res, starts):
            sl = slice(i0, i0 + rows_per_worker)
            pairs.append(({k: gpu[k][sl] for k in ("offR", "offA", "corr", "type")}, o))
        out[name] = _accuracy_blocks(pairs)
        out[name]["sample"] = f"{workers} x {rows_per_worker} grid rows spread over the grid, FP64 oracle, {wall:.1f} s"
    return out


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


def parity_other_configs(ctx):
    """Parity of the other tracking configurations against the FP64 oracle,
    recorded on the bench line: cfg1 (strack, 1024 x 2048 pair, W = 32, step
    16 x 8, the whole 124 x 119 grid, complex + amplitude fallback) and the
    cfg3 geometry (strackw, search window 224, edge pad 48, navg 2) on 240
    points spread over a 2000 x 4000 shear-zone pair."""
    from specklesource_b200 import abi, synth
    cores = os.cpu_count()
    out = {}
    s1, s2 = synth.small_pair(device="cuda", na=1024, nr=2048)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    g1 = dict(rStart=40, aStart=40, deltaR=16, deltaA=8, nR=124, nA=119, wR=32, wA=32, wRa=32, wAa=32)
    res = ctx.strack(abi.TrackParams(**g1), a, b)
    rows = (g1["nA"] + cores - 1) // cores
    blocks = [(i0, min(rows, g1["nA"] - i0), 0, g1["nR"]) for i0 in range(0, g1["nA"], rows)]
    r64, wall = _oracle_bands("strack", a, b, g1, blocks, 2 * 32 + 48, "f64")
    out["cfg1_strack_1024x2048_w32"] = dict(_accuracy(r64, blocks, res), oracle_s=wall)
    s1, s2 = synth.shear_pair(device="cuda", na=2000, nr=4000, seed=3)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    del s1, s2
    g3 = dict(rStart=160, aStart=160, deltaR=160, deltaA=140, nR=20, nA=12, wR=224, wA=224, wRa=224, wAa=224,
              edgePadR=48, edgePadA=48, navgR=2, navgA=2)
    res = ctx.strackw(abi.TrackParams(**g3), a, b)
    blocks = [(i, 1, 0, g3["nR"]) for i in range(g3["nA"])]
    r64, wall = _oracle_bands("strackw", a, b, g3, blocks, 224, "f64")
    out["cfg3_strackw_2000x4000_shear_w224"] = dict(_accuracy(r64, blocks, res), oracle_s=wall)
    return out


def throughput_other_configs(ctx, args):
    """Throughput of the other configurations, recorded on the default bench
    line so that the same run measures them: cfg1 (strack 1024 x 2048, W 32),
    cfg3 (strackw 8000 x 16000 shear, search 224), cfg4 (256 heterogeneous
    tiles + cullst) and cfg5 (serving), each with one warm-up pass and a short
    timed run.  A failure is recorded as a string and does not stop the line."""
    import copy
    import torch
    from specklesource_b200 import abi, synth
    out = {}
    try:
        s1, s2 = synth.small_pair(device="cuda", na=1024, nr=2048)
        g1 = abi.TrackParams(rStart=40, aStart=40, deltaR=16, deltaA=8, nR=124, nA=119, wR=32, wA=32, wRa=32,
                             wAa=32)
        ms = _time_calls(ctx, lambda: ctx.strack(g1, s1, s2), 20, 3)
        out["cfg1"] = {"workload": "strack 1024x2048 w32 step 16x8, complex + fallback, device images",
                       "patches_per_s": 124 * 119 / (np.median(ms) * 1e-3), "ms_per_call": float(np.median(ms))}
        del s1, s2
    except Exception as ex:  # recorded, not fatal
        out["cfg1"] = f"failed: {ex}"
    try:
        na, nr = 8000, 16000
        s1, s2 = synth.shear_pair(device="cuda", na=na, nr=nr, seed=3)
        g3 = abi.TrackParams(rStart=160, aStart=160, deltaR=32, deltaA=32, nR=(nr - 320) // 32 + 1,
                             nA=(na - 320) // 32 + 1, wR=224, wA=224, wRa=224, wAa=224, edgePadR=48, edgePadA=48,
                             navgR=2, navgA=2)
        ms = _time_calls(ctx, lambda: ctx.strackw(g3, s1, s2), 2, 1)
        n3 = g3.nR * g3.nA
        out["cfg3"] = {"workload": "strackw 8000x16000 shear, search 224, edge pad 48, step 32, navg 2",
                       "points": n3, "points_per_s": n3 / (np.median(ms) * 1e-3), "ms_per_call": float(np.median(ms))}
        del s1, s2
        torch.cuda.empty_cache()
    except Exception as ex:
        out["cfg3"] = f"failed: {ex}"
    for name, fn in (("cfg4", run_batched), ("cfg5", run_serving)):
        try:
            a2 = copy.copy(args)
            # two warm-up passes for cfg4: the slots' contexts reach their
            # buffer sizes (a reallocation waits for the whole device)
            a2.steps, a2.warmup = 1, 2 if name == "cfg4" else 1
            r = fn(a2)
            r.pop("clocks", None)
            out[name] = r
            torch.cuda.empty_cache()
        except Exception as ex:
            out[name] = f"failed: {ex}"
    return out


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


def bench_config(world):
    """The `config` of the bench line, shared by both arms."""
    img_bytes = 2 * NA * NR * 8
    return {"workload": f"strack {NA}x{NR} w64 step 24x6 ({N_A * N_R:,} patches, complex + amplitude fallback)",
            "parallelism": f"replicas x{world}", "l2": f"inputs {img_bytes / 1e9:.2f} GB > 126 MB L2, no flush"}


def run_reference(args):
    """The reference arm: the CPU restatement of the path on all host cores
    (the reference itself needs FFTW 2, Numerical Recipes and GDAL, absent
    here).  Each step tracks a bounded sample of the workload's grid rows;
    ms_per_step is that sample's measured time, not the whole grid's."""
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
    vals, secs = [], []
    cb = None
    for k in range(args.warmup + args.steps):
        rows = 1 if k < args.warmup else args.cpu_rows
        r = cpu_baseline(a, b, rows_per_worker=rows)
        if k >= args.warmup:
            vals.append(r["value"])
            secs.append(r["sample_s"])
            cb = r
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v,
            "unit": "patches/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * float(np.median(secs)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded speckle pair, no public dataset)",
            "config": bench_config(args.gpus),
            "step": {"what": "one bounded sample of the workload per step: the CPU restatement on "
                             f"{cb['cores']} processes x {args.cpu_rows} grid rows spread over the grid",
                     "sample_patches_per_step": cb["sample_patches"],
                     "ms_per_step_measured_on_sample": True,
                     "ms_full_grid_extrapolated": 1e3 * N_A * N_R / v},
            "cpu_baseline": dict(cb, value=v),
            "e2e": {"value": v, "unit": "patches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- other configurations
# Optional measurement modes for the benchmark's other configurations (not the
# default bench line): cfg1 (1024 x 2048, W=32, complex + amplitude fallback and
# amplitude only), cfg3 (strackw, 8000 x 16000 shear pair, search window 224,
# edge pad 48, step 32, 5 x 5 box smoothing) and cull (the cullst passes on an
# offsets grid of the default workload's size with 8 % outliers, 2 % NaN).

def _band_worker(args):
    fn, band1, band2, grid, precision = args
    sys.path.insert(0, ROOT)
    from oracle import oracle
    from specklesource_b200 import abi
    p = abi.TrackParams(**grid)
    t = time.time()
    o = getattr(oracle, fn)(p, band1, band2, precision=precision)
    return time.time() - t, grid["nA"] * grid["nR"], {k: o[k] for k in ("offR", "offA", "corr", "type")}


def _oracle_bands(fn, img1, img2, grid, row_blocks, margin, precision):
    """Oracle over blocks (i0, nrows, r0, ncols) of a grid, one spawned process
    per block, each given only the image band its windows reach."""
    import multiprocessing as mp
    jobs = []
    for i0, nrows, j0, ncols in row_blocks:
        a_lo = grid["aStart"] + i0 * grid["deltaA"] - margin
        a_hi = grid["aStart"] + (i0 + nrows - 1) * grid["deltaA"] + margin
        lo = max(0, a_lo)
        g = dict(grid, nA=nrows, nR=ncols, aStart=grid["aStart"] + i0 * grid["deltaA"] - lo,
                 rStart=grid["rStart"] + j0 * grid["deltaR"])
        jobs.append((fn, np.ascontiguousarray(img1[lo:a_hi]), np.ascontiguousarray(img2[lo:a_hi]), g, precision))
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(len(jobs)) as pool:
        res = pool.map(_band_worker, jobs)
    return res, time.time() - t0


def _accuracy(res, blocks, gpu):
    pairs = []
    for (_, _, o), (i0, nrows, j0, ncols) in zip(res, blocks):
        pairs.append(({k: gpu[k][i0:i0 + nrows, j0:j0 + ncols] for k in ("offR", "offA", "corr", "type")}, o))
    return _accuracy_blocks(pairs)


def _time_calls(ctx, call, steps, warmup):
    for _ in range(warmup):
        call()
    ms = []
    for _ in range(steps):
        call()
        ms.append(ctx.timing()["total"])
    return ms


def _plant_outliers(seed):
    """Injects 8 % uniform +-20 px outliers and 2 % NaN holes into matched points."""
    def inject(offR, offA, corr, mt):
        rng = np.random.default_rng(seed)
        ok = mt > 0
        m = ok & (rng.random(offR.shape) < 0.08)
        offR[m] += rng.uniform(-20, 20, m.sum()).astype(np.float32)
        offA[m] += rng.uniform(-20, 20, m.sum()).astype(np.float32)
        h = ok & (rng.random(offR.shape) < 0.02)
        offR[h] = np.nan
        offA[h] = np.nan
    return inject


def _tile_job(serve, abi, synth, torch, k, na, nr, w, radius, seed, cull=True, mode=None):
    """One synthetic tile job.  w <= 64: strack with complex window w (amplitude
    fallback on; mode "amplitude" runs -noComplex); w in (96, 128): strackw
    with search window w + 2 radius rounded to a supported size and edge pad
    radius.  Grid step w / 2, windows inside the tile."""
    s1, s2 = synth.make_pair(na, nr, seed,
                             dr=lambda y, x: 1.5 + 1.0 * torch.sin(2 * np.pi * x / 900),
                             da=lambda y, x: 0.5 * torch.cos(2 * np.pi * y / 700),
                             coherence=0.6, device="cuda")
    if w <= 64:
        W = w
        margin = W + 8
        step = max(8, W // 2)
        nR, nA = (nr - 2 * margin) // step + 1, (na - 2 * margin) // step + 1
        p = abi.TrackParams(rStart=margin, aStart=margin, deltaR=step, deltaA=step, nR=nR, nA=nA, wR=W, wA=W,
                            wRa=W, wAa=W, noComplex=int(mode == "amplitude"))
        kind = "strack"
    else:
        Ws = {96: 128, 128: 192}[w]
        pad = min(max(radius, 8), Ws // 2 - 24)  # strackw needs edgepad >= NFAST/4 = 5
        step = w // 2
        margin = Ws // 2 + 8
        nR, nA = (nr - 2 * margin) // step + 1, (na - 2 * margin) // step + 1
        p = abi.TrackParams(rStart=margin, aStart=margin, deltaR=step, deltaA=step, nR=nR, nA=nA, wR=w, wA=w,
                            wRa=Ws, wAa=Ws, edgePadR=pad, edgePadA=pad, navgR=2, navgA=2)
        kind = "strackw"
    if nR < 1 or nA < 1:
        return None
    cp = abi.CullParams(nR=nR, nA=nA, bR=5, bA=5, nGood=12, sR=3, sA=3, islandThresh=10) if cull else None
    return serve.Job(kind=kind, params=p, img1=s1, img2=s2, cull=cp, inject=_plant_outliers(seed) if cull else None,
                     tag=k)


def run_batched(args):
    """cfg4: 256 tiles (sides U[512, 4096], seeded) mixing windows
    {24, 32, 48, 64, 96, 128} and radii {4, 8, 16, 32}, all submitted at once
    to the job server; every offsets grid then goes through cullst (box 5,
    3 passes, 3x3 smoothing, islands 10) with 8 % outliers and 2 % NaN planted."""
    import torch
    from specklesource_b200 import abi, serve, synth
    rng = np.random.default_rng(4)
    jobs = []
    for k in range(256):
        na, nr = (int(x) for x in rng.integers(512, 4097, 2))
        w = int(rng.choice([24, 32, 48, 64, 96, 128]))
        radius = int(rng.choice([4, 8, 16, 32]))
        j = _tile_job(serve, abi, synth, torch, k, na, nr, w, radius, seed=400 + k)
        if j is not None:
            jobs.append(j)
    torch.cuda.synchronize()
    pts = sum(j.params.nR * j.params.nA for j in jobs)
    clocks = ClockSampler(0)
    with serve.JobServer(slots=args.slots, hbm_budget=120e9, max_batch=args.max_batch) as srv:
        # warm-up: the whole job set, so every slot holds its tables and buffers
        for _ in range(max(1, args.warmup)):
            [f.result() for f in [srv.submit(j) for j in jobs]]
        clocks.start()
        walls = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            for j in jobs:
                j.arrival = 0.0
            res = [f.result() for f in [srv.submit(j) for j in jobs]]
            walls.append(time.perf_counter() - t0)
        wall = float(np.median(walls))
        clk = clocks.stop()
        # the batched form: every strack tile in one sb_strack_batch call (stages
        # once per window group), strackw tiles and all culls on the server's slots
        from specklesource_b200 import runtime
        bctx = runtime.Context(0)
        st_jobs = [j for j in jobs if j.kind == "strack"]
        sw_jobs = [j for j in jobs if j.kind != "strack"]
        bwalls = []
        for rep in range(max(1, args.warmup) + max(1, args.steps)):
            t0 = time.perf_counter()
            futs = [srv.submit(j) for j in sw_jobs]
            bres = bctx.strack_batch([j.params for j in st_jobs], [j.img1 for j in st_jobs],
                                     [j.img2 for j in st_jobs])
            futs += [srv.submit(serve.Job(kind="cull", params=None, img1=(r["offR"], r["offA"], r["corr"], r["type"]),
                                          img2=None, cull=j.cull, inject=j.inject, tag=j.tag))
                     for j, r in zip(st_jobs, bres)]
            [f.result() for f in futs]
            if rep >= max(1, args.warmup):
                bwalls.append(time.perf_counter() - t0)
        bwall = float(np.median(bwalls))
        # breakdown, tracking only: the strack tiles on the server's slots
        # against one sb_strack_batch call, and the strackw tiles on the slots
        def _wall(fn):
            ts = []
            for rep in range(max(1, args.warmup) + max(1, args.steps)):
                t0 = time.perf_counter()
                fn()
                if rep >= max(1, args.warmup):
                    ts.append(time.perf_counter() - t0)
            return float(np.median(ts))
        st_track = [dataclasses.replace(j, cull=None, inject=None) for j in st_jobs]
        sw_track = [dataclasses.replace(j, cull=None, inject=None) for j in sw_jobs]
        t_st_srv = _wall(lambda: [f.result() for f in [srv.submit(j) for j in st_track]])
        t_st_batch = _wall(lambda: bctx.strack_batch([j.params for j in st_jobs], [j.img1 for j in st_jobs],
                                                     [j.img2 for j in st_jobs]))
        t_sw_srv = _wall(lambda: [f.result() for f in [srv.submit(j) for j in sw_track]])
        st_pts = sum(j.params.nR * j.params.nA for j in st_jobs)
        sw_pts = sum(j.params.nR * j.params.nA for j in sw_jobs)
        bctx.close()
    n_w = collections.Counter(("strack w%d" % j.params.wR) if j.kind == "strack" else
                              ("strackw w%d" % j.params.wRa) for j in jobs)
    matched = sum(int((r["track"]["type"] > 0).sum()) for r in res)
    return {"workload": f"cfg4 {len(jobs)} tiles 512-4096 px, windows 24-128, strack/strackw + cullst, "
                        f"{args.slots} server slots", "patches": pts, "value": pts / wall,
            "unit": "patches/s (tracking + culling, wall clock)", "wall_s": wall,
            "jobs_per_s": len(jobs) / wall, "matched_fraction": matched / pts, "mix": dict(n_w),
            "note": "jobs overlap across server slots (one CUDA stream each), a slot batching up to "
                    f"{args.max_batch} queued strack jobs of one window into one call; "
                    f"median wall of {len(walls)} passes after {max(1, args.warmup)} warm-up passes",
            "batched": {"value": pts / bwall, "wall_s": bwall, "strack_tiles_in_one_call": len(st_jobs),
                        "what": "strack tiles in one sb_strack_batch call (stages once per window group), strackw "
                                "tiles and every cull on the server's slots at the same time"},
            "tracking_only": {
                "strack_tiles": {"patches": st_pts, "server_s": t_st_srv, "batch_call_s": t_st_batch,
                                 "server_patches_per_s": st_pts / t_st_srv,
                                 "batch_patches_per_s": st_pts / t_st_batch},
                "strackw_tiles": {"points": sw_pts, "server_s": t_sw_srv, "points_per_s": sw_pts / t_sw_srv},
                "what": "no culling; median wall of the timed passes after the warm-up passes"},
            "clocks": clk}


def run_serving(args):
    """cfg5: Poisson arrivals (40 jobs/s, seeded) of track + cull jobs on pairs
    of 1024^2 - 8192^2 px (log-uniform), amplitude-only or complex mode,
    window 32 - 64 (strack's complex window limit; search radius follows the
    reference's acceptance rule |shift| < W/4), images resident in HBM,
    admitted against a 120 GB budget.  Reports jobs/s, patches/s and the
    arrival-to-completion latency percentiles."""
    import torch
    from specklesource_b200 import abi, serve, synth
    rng = np.random.default_rng(5)
    n_jobs = args.jobs
    # a pool of resident pairs to crop from (generating 8192^2 pairs per job
    # would time the generator, not the server)
    pool = {}
    for side in (1024, 2048, 4096, 8192):
        pool[side] = synth.make_pair(side, side, 500 + side,
                                     dr=lambda y, x: 1.5 + 1.0 * torch.sin(2 * np.pi * x / 900),
                                     da=lambda y, x: 0.5 * torch.cos(2 * np.pi * y / 700),
                                     coherence=0.6, device="cuda")
    jobs = []
    for k in range(n_jobs):
        side = int(np.exp(rng.uniform(np.log(1024), np.log(8192))))
        src = min(s for s in pool if s >= side)
        a, b = pool[src]
        mode = "amplitude" if rng.random() < 0.5 else "complex"
        W = int(rng.choice([32, 48, 64]))
        margin, step = W + 8, W // 2
        n = (side - 2 * margin) // step + 1
        p = abi.TrackParams(rStart=margin, aStart=margin, deltaR=step, deltaA=step, nR=n, nA=n, wR=W, wA=W, wRa=W,
                            wAa=W, noComplex=int(mode == "amplitude"))
        cp = abi.CullParams(nR=n, nA=n, bR=5, bA=5, nGood=12, sR=3, sA=3, islandThresh=10)
        jobs.append((serve.Job(kind="strack", params=p, img1=a[:side, :side].contiguous(),
                               img2=b[:side, :side].contiguous(), cull=cp, tag=k), side))
    torch.cuda.synchronize()
    gaps = rng.exponential(1.0 / 40.0, n_jobs)
    clocks = ClockSampler(0)
    with serve.JobServer(slots=args.slots, hbm_budget=120e9, max_batch=args.max_batch) as srv:
        # warm-up: the job set once, unpaced, so every slot's tables and
        # buffers exist (a long-running server's steady state)
        [f.result() for f in [srv.submit(j) for j, _ in jobs]]
        clocks.start()
        t0 = time.perf_counter()
        futs, t_next = [], t0
        for (j, _), g in zip(jobs, gaps):
            t_next += g
            while time.perf_counter() < t_next:
                time.sleep(min(0.002, max(0.0, t_next - time.perf_counter())))
            j.arrival = time.perf_counter()
            futs.append(srv.submit(j))
        res = [f.result() for f in futs]
        wall = max(r["end"] for r in res) - t0
        clk = clocks.stop()
        peak = srv.peak_bytes
    pts = sum(j.params.nR * j.params.nA for j, _ in jobs)
    slowest = [{"side": side, "mode": "amplitude" if j.params.noComplex else "complex", "W": j.params.wR,
                "points": j.params.nR * j.params.nA, "wait_ms": 1e3 * (r["start"] - r["arrival"]),
                "service_ms": 1e3 * (r["end"] - r["start"])}
               for (j, side), r in sorted(zip(jobs, res), key=lambda t: -(t[1]["end"] - t[1]["arrival"]))[:3]]
    return {"workload": f"cfg5 serving: {n_jobs} Poisson(40/s) track+cull jobs, 1024-8192 px, amplitude or "
                        f"complex, W 32-64, {args.slots} slots, 120 GB budget", "jobs": n_jobs,
            "value": n_jobs / wall, "unit": "jobs/s", "patches_per_s": pts / wall,
            "latency_ms": serve.latency_stats(res), "slowest_jobs": slowest, "offered_jobs_per_s": 40.0,
            "wall_s": wall,
            "peak_admitted_gb": peak / 1e9, "max_batch": args.max_batch,
            "batched_job_fraction": float(np.mean([r.get("batch", 1) > 1 for r in res])), "clocks": clk}


def run_dftgemm(args):
    """Comparator for the split-BF16 DFT-GEMM form of the complex stage's
    transforms: the 2-D forward DFTs of both 64 x 64 windows and the 128 x 128
    zero-padded inverse as real GEMMs on the tensor cores (cuBLAS through
    torch.matmul), each complex product in the real block form
    [[Re, -Im], [Im, Re]] and each GEMM as three bf16 products (hi*hi, hi*lo,
    lo*hi) accumulated in fp32.  Timed on a batch of patches with the data in
    HBM between the row and column GEMMs (a library GEMM cannot keep it on
    chip), extrapolated to the default workload's 1,955,217 patches, and set
    beside the FP32 complex stage, which does all of that plus the loads,
    Doppler, peak search and oversampling."""
    import torch
    W = 64
    B = args.batch

    def dft(n_out, n_in, sign, pad_to=None):
        k = torch.arange(n_out, dtype=torch.float64)[:, None]
        t = torch.arange(n_in, dtype=torch.float64)[None, :]
        if pad_to:  # zero-padded inverse: input bins at their padded positions
            t = torch.where(t < n_in // 2, t, t + (pad_to - n_in))
            n = pad_to
        else:
            n = n_in
        ang = sign * 2 * np.pi * k * t / n
        re, im = torch.cos(ang), torch.sin(ang)
        return torch.cat([torch.cat([re, -im], 1), torch.cat([im, re], 1)], 0).float().cuda()

    def split(m):
        hi = m.to(torch.bfloat16)
        lo = (m - hi.float()).to(torch.bfloat16)
        return hi, lo

    def gemm3(a, b):  # a: (M, K) fp32 matrix, b: (K, N) fp32
        ah, al = split(a)
        bh, bl = split(b)
        c = torch.matmul(ah, bh).float()
        c += torch.matmul(ah, bl).float()
        c += torch.matmul(al, bh).float()
        return c

    Fw = dft(W, W, -1.0)                 # (128, 128) forward 64-point DFT, real block form
    Iw = dft(2 * W, W, 1.0, pad_to=2 * W)  # (256, 128) zero-padded inverse 64 -> 128
    x = torch.randn(2 * W, W * 2 * B, device="cuda")  # both windows of B patches: [Re; Im] x (W columns)
    s = torch.randn(2 * W, W * B, device="cuda")
    torch.cuda.synchronize()

    def step():
        y = gemm3(Fw, x)                                   # forward along one axis
        y = y.reshape(2 * W, 2 * B, W).transpose(0, 2).reshape(2 * W, -1).contiguous()
        y = gemm3(Fw, y)                                   # forward along the other axis
        z = gemm3(Iw, s)                                   # padded inverse rows (64 -> 128)
        z = z.reshape(4 * W, B, W).permute(2, 1, 0).reshape(2 * W, -1).contiguous()
        z = gemm3(Iw, z)                                   # padded inverse columns
        return y, z

    for _ in range(2):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    full = N_A * N_R
    return {"workload": f"split-BF16 DFT-GEMM comparator: 64x64 forward x2 + 128x128 padded inverse per patch, "
                        f"batch {B} patches, cuBLAS bf16 (3 products, fp32 accumulate)",
            "ms_per_batch": ms, "ms_extrapolated_1955217_patches": ms * full / B,
            "transforms_only": True, "unit": "ms"}


def run_other(args):
    import torch
    from specklesource_b200 import abi, runtime, synth
    torch.cuda.set_device(0)
    ctx = runtime.Context(0)
    cores = os.cpu_count()
    clocks = ClockSampler(0)
    lines = []
    if args.workload == "cfg1":
        s1, s2 = synth.small_pair(device="cuda", na=1024, nr=2048)
        a, b = synth.to_numpy(s1), synth.to_numpy(s2)
        grid = dict(rStart=40, aStart=40, deltaR=16, deltaA=8, nR=124, nA=119, wR=32, wA=32, wRa=32, wAa=32)
        for variant, extra in (("complex + amplitude fallback", {}), ("amplitude only (-noComplex)",
                                                                     {"noComplex": 1})):
            g = dict(grid, **extra)
            p = abi.TrackParams(**g)
            clocks = ClockSampler(0)
            clocks.start()
            ms = _time_calls(ctx, lambda: ctx.strack(p, s1, s2), args.steps, args.warmup)
            clk = clocks.stop()
            st = ctx.stage_timing()
            res = ctx.strack(p, a, b)
            n = grid["nR"] * grid["nA"]
            rows = (grid["nA"] + cores - 1) // cores
            blocks = [(i0, min(rows, grid["nA"] - i0), 0, grid["nR"]) for i0 in range(0, grid["nA"], rows)]
            r32, w32 = _oracle_bands("strack", a, b, g, blocks, 2 * 32 + 48, "f32")
            r64, _ = _oracle_bands("strack", a, b, g, blocks, 2 * 32 + 48, "f64")
            cpu = n / max(r[0] for r in r32)
            lines.append({"workload": f"cfg1 strack 1024x2048 w32 step 16x8, {variant}", "patches": n,
                          "value": n / (np.median(ms) * 1e-3), "unit": "patches/s",
                          "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
                          "stages": st, "accuracy": _accuracy(r64, blocks, res),
                          "cpu_baseline": {"value": cpu, "unit": "patches/s", "cores": len(blocks), "kind": "port",
                                           "sample": "whole grid, f32 CPU restatement"},
                          "clocks": clk})
    elif args.workload == "amp64":
        # amplitude-only tracking at window 64 (small try 64, large try 128):
        # 2048 x 4096 pair, coherence 0.6, step 32
        s1, s2 = synth.make_pair(2048, 4096, 11, dr=lambda y, x: 1.5 + torch.sin(2 * np.pi * x / 900),
                                 da=lambda y, x: 0.5 * torch.cos(2 * np.pi * y / 700), coherence=0.6, device="cuda")
        a, b = synth.to_numpy(s1), synth.to_numpy(s2)
        Wa = 64
        grid = dict(rStart=2 * Wa, aStart=2 * Wa, deltaR=32, deltaA=32, nR=(4096 - 4 * Wa) // 32 + 1,
                    nA=(2048 - 4 * Wa) // 32 + 1, wR=Wa, wA=Wa, wRa=Wa, wAa=Wa, noComplex=1)
        p = abi.TrackParams(**grid)
        clocks.start()
        ms = _time_calls(ctx, lambda: ctx.strack(p, s1, s2), args.steps, args.warmup)
        clk = clocks.stop()
        st = ctx.stage_timing()
        res = ctx.strack(p, a, b)
        n = grid["nR"] * grid["nA"]
        step = max(1, grid["nA"] // cores)
        blocks = [(i0, 1, 0, grid["nR"]) for i0 in range(0, grid["nA"], step)][:cores]
        r64, _ = _oracle_bands("strack", a, b, grid, blocks, 4 * Wa + 48, "f64")
        lines.append({"workload": "amplitude-only strack 2048x4096 w64 step 32 (small try 64, large try 128)",
                      "patches": n, "value": n / (np.median(ms) * 1e-3), "unit": "patches/s",
                      "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
                      "stages": st, "accuracy": _accuracy(r64, blocks, res), "clocks": clk})
    elif args.workload in ("cfg3", "cfg3small"):
        na, nr = (8000, 16000) if args.workload == "cfg3" else (2000, 4000)
        s1, s2 = synth.shear_pair(device="cuda", na=na, nr=nr, seed=3)
        Wn = 224
        grid = dict(rStart=160, aStart=160, deltaR=32, deltaA=32, nR=(nr - 320) // 32 + 1, nA=(na - 320) // 32 + 1,
                    wR=Wn, wA=Wn, wRa=Wn, wAa=Wn, edgePadR=48, edgePadA=48, navgR=2, navgA=2)
        p = abi.TrackParams(**grid)
        clocks.start()
        ms = _time_calls(ctx, lambda: ctx.strackw(p, s1, s2), args.steps, args.warmup)
        clk = clocks.stop()
        res = ctx.strackw(p, s1, s2)
        res = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in res.items()}
        a, b = synth.to_numpy(s1), synth.to_numpy(s2)
        n = grid["nR"] * grid["nA"]
        # one grid row segment of 12 points per core, spread over the grid
        blocks = [((k * grid["nA"]) // cores, 1, (k * 37) % (grid["nR"] - 12), 12) for k in range(cores)]
        r32, _ = _oracle_bands("strackw", a, b, grid, blocks, Wn, "f32")
        r64, _ = _oracle_bands("strackw", a, b, grid, blocks, Wn, "f64")
        cpu = sum(r[1] for r in r32) / max(r[0] for r in r32)
        lines.append({"workload": f"cfg3 strackw {na}x{nr} shear, search 224, edge pad 48, step 32, navg 2",
                      "patches": n, "value": n / (np.median(ms) * 1e-3), "unit": "patches/s",
                      "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
                      "accuracy": _accuracy(r64, blocks, res),
                      "cpu_baseline": {"value": cpu, "unit": "patches/s", "cores": cores, "kind": "port",
                                       "sample": f"{cores} x 12 points spread over the grid, f32 CPU restatement"},
                      "clocks": clk})
    elif args.workload == "dftgemm":
        lines.append(run_dftgemm(args))
    elif args.workload in ("cfg4", "cfg5"):
        lines.append(run_batched(args) if args.workload == "cfg4" else run_serving(args))
    elif args.workload == "cull":
        from oracle import oracle
        nA, nR = N_A, N_R
        offR, offA, corr, mt = synth.offsets_field(nA, nR, 4)
        cp = abi.CullParams(nR=nR, nA=nA, bR=5, bA=5, nGood=12, sR=3, sA=3, islandThresh=10, nCullPasses=3)
        clocks.start()
        ms = _time_calls(ctx, lambda: ctx.cull(cp, offR, offA, corr, mt), args.steps, args.warmup)
        clk = clocks.stop()
        g = ctx.cull(cp, offR, offA, corr, mt)
        t = time.time()
        o = oracle.cull(cp, offR, offA, corr, mt)
        cpu_s = time.time() - t
        keep = {k: bool(np.array_equal(g[k], o[k], equal_nan=True)) for k in ("offR", "offA", "type")}
        lines.append({"workload": f"cull {nA}x{nR} grid, 8% outliers, 2% NaN, box 5, 3 passes, smooth 3x3, "
                                  "islands 10", "points": nA * nR,
                      "value": nA * nR / (np.median(ms) * 1e-3), "unit": "grid points/s",
                      "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
                      "keep_mask_bit_exact": keep,
                      "cpu_baseline": {"value": nA * nR / cpu_s, "unit": "grid points/s", "cores": 1,
                                       "kind": "port", "sample": "whole grid, FP64 CPU restatement"},
                      "clocks": clk})
    for ln in lines:
        print(json.dumps(dict(ln, n_gpus=1, steps=args.steps, warmup=args.warmup, dtype="f32",
                              data="synthetic (seeded)")))
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-rows", type=int, default=32, help="grid rows per CPU process in the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32-peak", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP64-oracle check of a row sample")
    ap.add_argument("--form", default="fp32", choices=["fp32", "split-bf16"],
                    help="transform form of the complex stage timed for the headline value; the other form is "
                         "measured beside it")
    ap.add_argument("--no-other-form", action="store_true", help="skip measuring the other transform form")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the cfg1/cfg3/cfg4/cfg5 throughput block of the default line")
    ap.add_argument("--slots", type=int, default=4, help="job-server slots for --workload cfg4/cfg5")
    ap.add_argument("--jobs", type=int, default=200, help="jobs offered in --workload cfg5")
    ap.add_argument("--max-batch", type=int, default=1,
                    help="job server: queued strack jobs of one window that may share one sb_strack_batch call "
                         "(cfg4/cfg5; 1: every job its own call -- batches of varying size grow the contexts' "
                         "buffers while timed)")
    ap.add_argument("--batch", type=int, default=32768, help="patches per batch in --workload dftgemm")
    ap.add_argument("--workload", default="large",
                    choices=["large", "small", "cfg1", "cfg3", "cfg3small", "cfg4", "cfg5", "cull", "dftgemm", "amp64"],
                    help="small: 2400x4800 profiling case of the same generator; cfg1 / cfg3 / cull: the "
                         "other configurations (one JSON line each, not the bench line); cfg3small: the cfg3 "
                         "geometry on a 2000x4000 pair (profiling case); amp64: amplitude-only tracking at "
                         "window 64")
    args = ap.parse_args()
    if args.workload == "small":
        use_small_workload()
    if args.workload in ("cfg1", "cfg3", "cfg3small", "cfg4", "cfg5", "cull", "dftgemm", "amp64"):
        return run_other(args)
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

    from specklesource_b200 import abi
    ctx = runtime.Context(local)
    forms = {"fp32": abi.SB_FORM_FP32, "split-bf16": abi.SB_FORM_SPLIT_BF16}
    ctx.set_form(forms[args.form])
    p = track_params()
    s1, s2 = synth.large_pair(device="cuda", na=NA, nr=NR, seed=replica_seed(rank))
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
    ms_step = max_over_ranks(torch, tot_ms / args.steps, world, "cuda")
    value = job_rate(world, n_pts, ms_step)

    form_ran = ctx.last_form()
    outputs = {args.form: {k: out[k].cpu().numpy() for k in ("offR", "offA", "corr", "type")}}
    form_stats = {args.form: {"ms_per_call": ms_step, "patches_per_s": value,
                              "cmplx_ms": float(np.mean([s_["cmplx_ms"] for s_ in stages])),
                              "ran": "split-bf16" if form_ran == abi.SB_FORM_SPLIT_BF16 else "fp32"}}
    if not args.no_other_form:
        other = "split-bf16" if args.form == "fp32" else "fp32"
        ctx.set_form(forms[other])
        for _ in range(max(2, args.warmup)):
            step_dev()
        barrier()
        o_ms, o_cm = [], []
        for _ in range(args.steps):
            t, st, _ = step_dev()
            o_ms.append(t)
            o_cm.append(st["cmplx_ms"])
        barrier()
        om = max_over_ranks(torch, float(np.median(o_ms)), world, "cuda")
        form_stats[other] = {"ms_per_call": om, "patches_per_s": job_rate(world, N_A * N_R, om),
                             "cmplx_ms": float(np.median(o_cm)), "timing": f"median of {args.steps} calls",
                             "ran": "split-bf16" if ctx.last_form() == abi.SB_FORM_SPLIT_BF16 else "fp32"}
        outputs[other] = {k: out[k].cpu().numpy() for k in ("offR", "offA", "corr", "type")}
        ctx.set_form(forms[args.form])

    # ---- roofline of the dominant kernel (complex stage: FP32 CUDA cores, or
    # the tensor cores for the split-BF16 form)
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
        e_ms = max_over_ranks(torch, e_ms / args.steps, world, "cuda")
        e2e = {"value": job_rate(world, n_pts, e_ms), "unit": "patches/s", "h2d_bytes_per_step": img_bytes,
               "d2h_bytes_per_step": n_pts * (4 * 4 + 1), "ms_per_step": e_ms,
               "match_fraction": float((hout["type"] > 0).mean())}

    cpu, acc, parity = None, None, None
    if rank == 0 and world == 1 and not (args.no_cpu_baseline and args.no_accuracy):
        a = synth.to_numpy(s1)
        b = synth.to_numpy(s2)
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(a, b, rows_per_worker=args.cpu_rows)
        if not args.no_accuracy:
            acc_forms = accuracy_vs_fp64_forms(a, b, outputs)
            acc = acc_forms[args.form]
            for name, st_ in form_stats.items():
                st_["accuracy"] = acc_forms[name]
            del a, b
            parity = parity_other_configs(ctx)
    others = None
    if rank == 0 and world == 1 and args.workload == "large" and not args.no_other_configs:
        others = throughput_other_configs(ctx, args)
    if args.form == "split-bf16":
        # the split-BF16 kernel is bound by the tensor pipe: GEMM flops per patch
        # = 6 passes x 3 products x 2 x 128 x 128 x 128 (real block form)
        key = f"strack_cmplx_tc_w64_{NA}x{NR}"
        traffic = measured_traffic(key)
        gemm = 6 * 3 * 2.0 * 128 ** 3
        ach = st0["n_cmplx"] * gemm / (cm_ms * 1e-3) / 1e12
        tpk = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
        roofline = {
            "bound": "tensor", "achieved": ach, "peak": tpk, "unit": "TFLOP/s", "frac": ach / tpk,
            "peak_source": f"MEASURED_PEAKS.json bf16 dense, sustained ({src}); the complex stage runs inside "
                           "back-to-back calls",
            "gemm_flops_per_patch": gemm, "alg_flops_per_patch": ALG_CMPLX,
            "alg_tflops": ach_tflops, "alg_frac_of_fp32": ach_tflops / fp32,
            "traffic": traffic,
            "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, profiles/{key}.md"
                              if traffic else "no committed capture for this workload",
            "launch_patches": min(n_pts, PEAK_CHUNK), "launches_per_call": -(-n_pts // PEAK_CHUNK),
            "alg_bytes_per_launch": int((img_bytes + n_pts * (4 * 4 + 1)) * min(n_pts, PEAK_CHUNK) / n_pts),
            "kernel": "strack_cmplx_tc_kernel (tcgen05, M128 N64 K16 bf16, 144 MMAs per patch)",
            "hbm": {"achieved_gbs": img_bytes / (cm_ms * 1e-3) / 1e9, "peak_gbs": peaks.get("hbm_gbs"),
                    "peak_source": src},
        }
    else:
        key = f"strack_cmplx_w64_{NA}x{NR}"
        traffic = measured_traffic(key)
        roofline = {
            "bound": "fp32", "achieved": ach_tflops, "peak": fp32, "unit": "TFLOP/s",
            "frac": ach_tflops / fp32,
            "traffic": traffic,
            "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, profiles/{key}.md"
                              if traffic else "no committed capture for this workload",
            "launch_patches": min(n_pts, PEAK_CHUNK),
            "launches_per_call": -(-n_pts // PEAK_CHUNK),
            "alg_bytes_per_launch": int((img_bytes + n_pts * (4 * 4 + 1)) * min(n_pts, PEAK_CHUNK) / n_pts),
            "kernel": "strack_cmplx_kernel<64,256>",
            "alg_flops_per_patch": ALG_CMPLX,
            "peak_source": "cuBLAS SGEMM 8192^3 (TF32 off) measured in this run",
            "hbm": {"achieved_gbs": (img_bytes) / (cm_ms * 1e-3) / 1e9, "peak_gbs": peaks.get("hbm_gbs"),
                    "peak_source": src},
        }

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value, "unit": "patches/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded speckle pair, no public dataset)",
            "config": bench_config(world),
            "e2e": e2e,
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                           "what": "one sb_strack call over the whole grid, images resident"},
            "accuracy": acc,
            "parity_other_configs": parity,
            "other_configs": others,
            "gpu_launches": launches,
            "stages": {k: float(np.mean([s[k] for s in stages])) for k in stages[-1]},
            "form": args.form,
            "forms": form_stats,
            "roofline": roofline,
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
