"""Autotuner of the strack kernels' launch shapes, per window-size bucket.

    python -m specklesource_b200.autotune [--out specklesource_b200/tuning.json]

For every bucket it times the candidates on a synthetic pair of the
benchmark's generator (device-resident, the stage isolated by its own
CUDA-event timing, median of `reps` calls after a warm-up call):

  * FP32 complex stage, windows 16, 24, 32, 48, 64: both compiled thread
    counts x every resident CTA count per SM (amplitude tries off);
  * split-BF16 complex stage, window 64: 1 or 2 CTAs per SM;
  * shared-memory amplitude try, windows 16, 24, 32, 48: every resident CTA
    count per SM (-noComplex, one try; window 64 fits one CTA per SM, so
    there is nothing to choose).

and writes the fastest shape per bucket, with every candidate's time, to a
JSON table.  runtime.Context applies the table of the device it runs on
(sb_set_tuning) when it is created; results do not depend on the CTA count,
and a thread count changes only the order of float partial sums of the
patch powers.
"""
import argparse
import json
import os
import time

import numpy as np

from . import abi, runtime, synth

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tuning.json")

COMPLEX_THREADS = {16: (64, 128), 24: (96, 192), 32: (256, 128), 48: (192, 384), 64: (256, 512)}
KERNEL_IDS = {"complex": abi.SB_TUNE_COMPLEX, "complex_tc": abi.SB_TUNE_COMPLEX_TC,
              "amplitude": abi.SB_TUNE_AMPLITUDE}


def _grid(W, na, nr, **kw):
    step = max(8, W // 2)
    m = W + 8
    return abi.TrackParams(rStart=m, aStart=m, deltaR=step, deltaA=step, nR=(nr - 2 * m) // step + 1,
                           nA=(na - 2 * m) // step + 1, wR=W, wA=W, wRa=W, wAa=W, **kw)


def _time(ctx, p, s1, s2, key, reps):
    ctx.strack(p, s1, s2)
    ms = []
    for _ in range(reps):
        ctx.strack(p, s1, s2)
        ms.append(ctx.stage_timing()[key])
    return float(np.median(ms))


def _try_shapes(ctx, kernel, W, threads_list, p, s1, s2, key, reps):
    cands = []
    for threads in threads_list:
        for ctas in range(1, 5):
            rc = ctx.lib.sb_set_tuning(ctx.h, KERNEL_IDS[kernel], W, threads, ctas)
            if rc != abi.SB_OK:
                break  # above the resident maximum
            cands.append({"threads": threads, "ctas_per_sm": ctas, "ms": _time(ctx, p, s1, s2, key, reps)})
    ctx.lib.sb_set_tuning(ctx.h, KERNEL_IDS[kernel], W, 0, 0)
    best = min(cands, key=lambda c: c["ms"])
    return dict(kernel=kernel, window=W, threads=best["threads"], ctas_per_sm=best["ctas_per_sm"],
                ms=best["ms"], candidates=cands)


def tune(device=0, reps=3, na=2048, nr=4096):
    import torch
    ctx = runtime.Context(device, tuning=False)
    s1, s2 = synth.large_pair(device="cuda", na=na, nr=nr, seed=11)
    torch.cuda.synchronize()
    entries = []
    for W, ths in COMPLEX_THREADS.items():
        p = _grid(W, na, nr, maxTries=0)
        entries.append(_try_shapes(ctx, "complex", W, ths, p, s1, s2, "cmplx_ms", reps))
    ctx.set_form(abi.SB_FORM_SPLIT_BF16)
    entries.append(_try_shapes(ctx, "complex_tc", 64, (0,), _grid(64, na, nr, maxTries=0), s1, s2, "cmplx_ms",
                               reps))
    ctx.set_form(abi.SB_FORM_FP32)
    for W in (16, 24, 32, 48):
        p = _grid(W, na, nr, noComplex=1, maxTries=1)
        entries.append(_try_shapes(ctx, "amplitude", W, (0,), p, s1, s2, "amp_small_ms", reps))
    ctx.close()
    return {"device": torch.cuda.get_device_name(device), "sm_count": torch.cuda.get_device_properties(device)
            .multi_processor_count, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
            "workload": f"synthetic {na} x {nr} pair of the benchmark generator, step W/2, median of {reps} calls",
            "entries": entries}


def apply(ctx, table):
    """Applies a tuning table (dict) to a runtime.Context; entries the library
    refuses (e.g. a thread count no longer compiled) are skipped.  Returns the
    number applied."""
    n = 0
    for e in table.get("entries", []):
        kid = KERNEL_IDS.get(e.get("kernel"))
        if kid is None:
            continue
        if ctx.lib.sb_set_tuning(ctx.h, kid, int(e["window"]), int(e.get("threads", 0)),
                                 int(e.get("ctas_per_sm", 0))) == abi.SB_OK:
            n += 1
    return n


def load(path=DEFAULT_TABLE):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    t = tune(reps=args.reps)
    with open(args.out, "w") as f:
        json.dump(t, f, indent=1)
    for e in t["entries"]:
        print(f"{e['kernel']:>10} W={e['window']:3d}: threads {e['threads']} ctas/SM {e['ctas_per_sm']} "
              f"{e['ms']:.3f} ms")


if __name__ == "__main__":
    main()
