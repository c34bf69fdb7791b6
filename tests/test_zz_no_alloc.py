"""The allocation-free entry point sb_amp_match_noalloc against sb_strack.

sb_amp_match_noalloc serves callers that may not allocate device memory
while they run (an application that has reserved the GPU memory for its own
pool, or a latency-critical loop where cudaMalloc would synchronise).  This
test calls it through the C ABI on the patches of an amplitude-only strack
grid and checks, on two calls in a row (the fixed workspace keeps the first
call's contents), that it reproduces the amplitude try of the existing entry
point within the tracking tolerance of the other GPU tests.  It lives in its
own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

from specklesource_b200 import abi, synth

from .parity import compare_track

pytestmark = pytest.mark.gpu

NOVER, OS = 12, 2


def _amp_result(cmax, imax, jmax, hd, r_shift_amp, a_shift_amp, wa):
    """Output grids of a single amplitude try (speckleTrack.c:270-323, s = 1)."""
    inv = 1.0 / np.float32(NOVER)
    r1 = ((jmax.astype(np.float32).astype(np.float64) - wa * 0.5 * OS * NOVER) * inv / OS).astype(np.float32)
    a1 = ((imax.astype(np.float32).astype(np.float64) - wa * 0.5 * OS * NOVER) * inv / OS).astype(np.float32)
    good = (hd == 1) & (np.abs(r1.astype(np.float64)) < 0.15 * wa * OS) & \
        (np.abs(a1.astype(np.float64)) < 0.15 * wa * OS) & (cmax > 0.07)
    offR = np.where(good, (r_shift_amp - r1).astype(np.float32), np.float32(-2e9)).astype(np.float32)
    offA = np.where(good, (a_shift_amp - a1).astype(np.float32), np.float32(-2e9)).astype(np.float32)
    corr = np.where(hd == 1, cmax, 0.0).astype(np.float32)
    return {"offR": offR, "offA": offA, "corr": corr, "type": np.where(good, 2, 0).astype(np.uint8)}


def test_noalloc_amplitude_try_matches_strack():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from specklesource_b200 import build, runtime
    build.build()
    wa = 32
    s1, s2 = synth.small_pair(na=256, nr=512)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    p = abi.TrackParams(rStart=40, aStart=40, deltaR=16, deltaA=16, nR=27, nA=12, wR=wa, wA=wa, wRa=wa, wAa=wa,
                        noComplex=1, maxTries=1)
    with runtime.Context(0) as ctx:
        ref = ctx.strack(p, a, b)
        # windows of the small amplitude try (zero initial shift: r2 = r1, a2 = a1)
        jj, ii = np.meshgrid(np.arange(p.nR), np.arange(p.nA))
        r1 = p.rStart + jj * p.deltaR - p.wR // 2
        a1 = p.aStart + ii * p.deltaA - p.wA // 2
        inb = (r1 > 0) & (r1 + wa < a.shape[1]) & (a1 > 0) & (a1 + wa < a.shape[0])
        sel = np.flatnonzero(inb.ravel())
        P1 = np.stack([a[a1.flat[k]:a1.flat[k] + wa, r1.flat[k]:r1.flat[k] + wa] for k in sel])
        P2 = np.stack([b[a1.flat[k]:a1.flat[k] + wa, r1.flat[k]:r1.flat[k] + wa] for k in sel])
        t1 = torch.from_numpy(np.ascontiguousarray(P1)).cuda()
        t2 = torch.from_numpy(np.ascontiguousarray(P2)).cuda()
        n = len(sel)
        outs = []
        for _ in range(2):
            cmax = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
            imax = torch.zeros(n, dtype=torch.int32, device="cuda")
            jmax = torch.zeros(n, dtype=torch.int32, device="cuda")
            hd = torch.zeros(n, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            rc = ctx.lib.sb_amp_match_noalloc(ctx.h, t1.data_ptr(), t2.data_ptr(), n, wa, None, cmax.data_ptr(),
                                              imax.data_ptr(), jmax.data_ptr(), hd.data_ptr())
            assert rc == abi.SB_OK, ctx.lib.sb_last_error(ctx.h)
            outs.append((cmax.cpu().numpy(), imax.cpu().numpy(), jmax.cpu().numpy(), hd.cpu().numpy()))
        # sizes beyond the static workspace's maximum are refused, not run
        rc = ctx.lib.sb_amp_match_noalloc(ctx.h, t1.data_ptr(), t2.data_ptr(), n, 128, None, cmax.data_ptr(),
                                          imax.data_ptr(), jmax.data_ptr(), hd.data_ptr())
        assert rc == abi.SB_ERR_ARG and b"maximum" in ctx.lib.sb_last_error(ctx.h)
    for cm, im, jm, h in outs:
        got = {k: ref[k].copy() for k in ("offR", "offA", "corr", "type")}
        res = _amp_result(cm, im, jm, h, np.float32(0.0), np.float32(0.0), wa)
        for k in got:
            got[k].flat[sel] = res[k]
        st = compare_track(got, {k: ref[k] for k in got})
        assert st["pass"], st
        assert st["n_match_oracle"] > 100
    assert np.array_equal(outs[0][1], outs[1][1]) and np.array_equal(outs[0][2], outs[1][2])
