"""The allocation-free entry point sb_amp_match_noalloc against the FP64 oracle.

sb_amp_match_noalloc serves callers that may not allocate device memory
while they run: an application that has reserved the GPU's memory for its own
pool, or a latency-critical loop in which cudaMalloc would synchronise the
device.  These tests call it through the C ABI on the patches of an
amplitude-only strack grid, for every supported window, and check on two
calls in a row (the fixed workspace keeps the first call's contents) that it
reproduces the oracle's amplitude try within the tracking tolerance of the
other GPU tests, that a caller-supplied roll (the oracle's Doppler estimate,
also shifted by +-wa) gives the same result as letting the kernel estimate
it, and that a call changes the device's free memory by nothing.  The file
is collected last.
"""

import numpy as np
import pytest

from oracle import oracle
from specklesource_b200 import abi, synth

from .parity import compare_track

pytestmark = pytest.mark.gpu

NOVER, OS = 12, 2


def _amp_result(cmax, imax, jmax, hd, wa):
    """Output grids of a single amplitude try at zero initial shift
    (speckleTrack.c:270-323, s = 1)."""
    inv = 1.0 / np.float32(NOVER)
    r1 = ((jmax.astype(np.float32).astype(np.float64) - wa * 0.5 * OS * NOVER) * inv / OS).astype(np.float32)
    a1 = ((imax.astype(np.float32).astype(np.float64) - wa * 0.5 * OS * NOVER) * inv / OS).astype(np.float32)
    good = (hd == 1) & (np.abs(r1.astype(np.float64)) < 0.15 * wa * OS) & \
        (np.abs(a1.astype(np.float64)) < 0.15 * wa * OS) & (cmax > 0.07)
    offR = np.where(good, (np.float32(0.0) - r1).astype(np.float32), np.float32(-2e9)).astype(np.float32)
    offA = np.where(good, (np.float32(0.0) - a1).astype(np.float32), np.float32(-2e9)).astype(np.float32)
    corr = np.where(hd == 1, cmax, 0.0).astype(np.float32)
    return {"offR": offR, "offA": offA, "corr": corr, "type": np.where(good, 2, 0).astype(np.uint8)}


@pytest.fixture(scope="module")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from specklesource_b200 import build, runtime
    build.build()
    c = runtime.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def pair():
    s1, s2 = synth.small_pair(na=256, nr=512)
    return synth.to_numpy(s1), synth.to_numpy(s2)


def _call(ctx, t1, t2, n, wa, az):
    import torch
    cmax = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
    imax = torch.full((n,), 5, dtype=torch.int32, device="cuda")
    jmax = torch.full((n,), 5, dtype=torch.int32, device="cuda")
    hd = torch.full((n,), 9, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = ctx.lib.sb_amp_match_noalloc(ctx.h, t1.data_ptr(), t2.data_ptr(), n, wa,
                                      None if az is None else az.data_ptr(), cmax.data_ptr(), imax.data_ptr(),
                                      jmax.data_ptr(), hd.data_ptr())
    assert rc == abi.SB_OK, ctx.lib.sb_last_error(ctx.h)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return (cmax.cpu().numpy(), imax.cpu().numpy(), jmax.cpu().numpy(), hd.cpu().numpy()), free0 - free1


@pytest.mark.parametrize("wa", [16, 24, 32, 48, 64])
def test_noalloc_amplitude_try_matches_oracle(ctx, pair, wa):
    import torch
    a, b = pair
    step = max(16, wa // 2)
    nR, nA = (512 - 80) // step, (256 - 80) // step
    p = abi.TrackParams(rStart=40, aStart=40, deltaR=step, deltaA=step, nR=nR, nA=nA, wR=wa, wA=wa, wRa=wa,
                        wAa=wa, noComplex=1, maxTries=1)
    orc = oracle.strack(p, a, b)
    # windows of the small amplitude try (zero initial shift: r2 = r1, a2 = a1)
    jj, ii = np.meshgrid(np.arange(nR), np.arange(nA))
    r1 = p.rStart + jj * p.deltaR - wa // 2
    a1 = p.aStart + ii * p.deltaA - wa // 2
    inb = (r1 > 0) & (r1 + wa < a.shape[1]) & (a1 > 0) & (a1 + wa < a.shape[0])
    sel = np.flatnonzero(inb.ravel())
    P1 = np.ascontiguousarray(np.stack([a[a1.flat[k]:a1.flat[k] + wa, r1.flat[k]:r1.flat[k] + wa] for k in sel]))
    P2 = np.ascontiguousarray(np.stack([b[a1.flat[k]:a1.flat[k] + wa, r1.flat[k]:r1.flat[k] + wa] for k in sel]))
    n = len(sel)
    # the roll estDopCarrier1 gives for each pair (what the kernel estimates when azShift is NULL)
    az = np.array([oracle.est_dop_carrier(P1[k], P2[k], wa) for k in range(n)], np.int32)
    t1 = torch.from_numpy(P1).cuda()
    t2 = torch.from_numpy(P2).cuda()
    outs = []
    for _ in range(2):  # two calls in a row: the workspace keeps the first call's contents
        o, dfree = _call(ctx, t1, t2, n, wa, None)
        assert dfree == 0, f"a call changed the device's free memory by {dfree} bytes"
        outs.append(o)
    rolls = [torch.from_numpy(az + sh).cuda() for sh in (0, wa, -wa)]
    for r in rolls:
        o, dfree = _call(ctx, t1, t2, n, wa, r)
        assert dfree == 0
        for x, y in zip(o, outs[0]):
            assert np.array_equal(x, y), "a caller-supplied roll (mod wa) changed the result"
    for cm, im, jm, h in outs:
        got = {k: orc[k].copy() for k in ("offR", "offA", "corr", "type")}
        res = _amp_result(cm, im, jm, h, wa)
        for k in got:
            got[k].flat[sel] = res[k]
        st = compare_track(got, {k: orc[k] for k in got})
        print(wa, n, st)
        assert st["pass"], st
        assert st["n_match_oracle"] >= 0.3 * n
    for x, y in zip(outs[0], outs[1]):
        assert np.array_equal(x, y)


def test_noalloc_rejects_sizes_beyond_its_workspace(ctx):
    import torch
    n = 4
    t = torch.zeros((n, 128, 128), dtype=torch.complex64, device="cuda")
    cmax = torch.zeros(n, dtype=torch.float64, device="cuda")
    i32 = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc = ctx.lib.sb_amp_match_noalloc(ctx.h, t.data_ptr(), t.data_ptr(), n, 128, None, cmax.data_ptr(),
                                      i32.data_ptr(), i32.data_ptr(), i32.data_ptr())
    assert rc == abi.SB_ERR_ARG and b"maximum" in ctx.lib.sb_last_error(ctx.h)
    rc = ctx.lib.sb_amp_match_noalloc(ctx.h, t.data_ptr(), t.data_ptr(), n, 40, None, cmax.data_ptr(),
                                      i32.data_ptr(), i32.data_ptr(), i32.data_ptr())
    assert rc == abi.SB_ERR_ARG
    rc = ctx.lib.sb_amp_match_noalloc(ctx.h, t.data_ptr(), t.data_ptr(), 0, 32, None, cmax.data_ptr(),
                                      i32.data_ptr(), i32.data_ptr(), i32.data_ptr())
    assert rc == abi.SB_ERR_ARG
