"""strack on the GPU (through the C ABI) against the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle
from specklesource_b200 import abi, synth

from .parity import compare_track

pytestmark = pytest.mark.gpu


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
def pair_1k():
    s1, s2 = synth.small_pair(na=1024, nr=2048)
    return synth.to_numpy(s1), synth.to_numpy(s2)


def _p(**kw):
    base = dict(rStart=40, aStart=40, deltaR=16, deltaA=8, nR=27, nA=25, wR=32, wA=32, wRa=32, wAa=32)
    base.update(kw)
    return abi.TrackParams(**base)


def _check(ctx, p, a, b, **kw):
    g = ctx.strack(p, a, b)
    o = oracle.strack(p, a, b)
    st = compare_track(g, o, **kw)
    print(st, g["stats"], o["stats"])
    assert st["pass"], st
    return g, o, st


def test_complex_default_small(ctx, small_pair_np):
    a, b = small_pair_np
    g, o, st = _check(ctx, _p(), a, b)
    assert st["n_match_oracle"] > 500
    assert ctx.launch_count() >= 3


def test_config1_full_grid(ctx, pair_1k):
    a, b = pair_1k
    p = _p(nR=124, nA=119)
    g, o, st = _check(ctx, p, a, b)
    for k in ("nComplex", "nAmp", "nAmpL"):
        assert abs(g["stats"][k] - o["stats"][k]) <= max(2, 0.005 * o["stats"]["nAttempted"])
    ok = (g["type"] > 0) & (o["type"] > 0)
    azd_rel = np.abs(g["azd"][ok] - o["azd"][ok]) / np.abs(o["azd"][ok])
    assert np.percentile(azd_rel, 99) < 1e-2


def test_amplitude_only(ctx, small_pair_np):
    a, b = small_pair_np
    g, o, st = _check(ctx, _p(noComplex=1), a, b)
    assert (o["type"] == abi.SB_AMPMATCH).sum() > 300


def test_no_hanning_single_amp(ctx, small_pair_np):
    a, b = small_pair_np
    _check(ctx, _p(hanningFlag=0, maxTries=1), a, b)


def test_window_64(ctx, pair_1k):
    a, b = pair_1k
    p = _p(wR=64, wA=64, wRa=64, wAa=64, deltaR=24, deltaA=24, nR=40, nA=20, rStart=64, aStart=64)
    _check(ctx, p, a, b)


def test_amplitude_only_window_64(ctx, pair_1k):
    """Amplitude tries at window 64: the small try in the lean shared-memory
    layout (tables read from global memory), the large one (128) staged."""
    a, b = pair_1k
    p = _p(noComplex=1, wR=64, wA=64, wRa=64, wAa=64, deltaR=24, deltaA=24, nR=40, nA=20, rStart=64, aStart=64)
    g, o, st = _check(ctx, p, a, b)
    assert (o["type"] == abi.SB_AMPMATCH).sum() > 300


def test_low_coherence_exercises_fallbacks(ctx):
    s1, s2 = synth.make_pair(512, 512, 21, dr=lambda y, x: 1.3 + 0 * x, da=lambda y, x: -0.6 + 0 * y,
                             coherence=0.25)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    p = _p(rStart=72, aStart=72, nR=24, nA=24, deltaR=16, deltaA=16)
    g, o, st = _check(ctx, p, a, b)
    assert o["stats"]["nAmp"] + o["stats"]["nAmpL"] > 0


def test_big_endian_and_int16_inputs(ctx, small_pair_np):
    a, b = small_pair_np
    p = _p()
    g1 = ctx.strack(p, a, b)
    g2 = ctx.strack(p, a.astype(">c8"), b.astype(">c8"))
    for k in ("offR", "offA", "corr", "type"):
        assert np.array_equal(g1[k], g2[k])
    scale = 3000.0
    ai = np.stack([np.round(a.real * scale), np.round(a.imag * scale)], -1).astype(np.int16)
    bi = np.stack([np.round(b.real * scale), np.round(b.imag * scale)], -1).astype(np.int16)
    gi = ctx.strack(p, ai, bi)
    oi = oracle.strack(p, ai, bi)
    st = compare_track(gi, oi)
    assert st["pass"], st
    gm = ctx.strack(p, ai.astype(">i2"), bi.astype(">i2"))
    assert np.array_equal(gm["offR"], gi["offR"])


def test_mask_and_offset_grid(ctx, small_pair_np):
    a, b = small_pair_np
    rng = np.random.default_rng(5)
    mask = (rng.random((16, 32)) > 0.3).astype(np.uint8)
    grid = {"nr": 20, "na": 12, "r0": 0.0, "a0": 0.0, "deltaR": 32.0, "deltaA": 32.0,
            "dr": np.full((12, 20), 2.0, np.float32), "da": np.full((12, 20), 0.4, np.float32)}
    grid["dr"][3:5, 3:6] = -2e9  # holes: the reference keeps the previous point's r2/a2
    p = _p(mask={"r0": 0, "a0": 0, "nr": 32, "na": 16, "nrl": 16, "nal": 16, "mask": mask},
           polyShift=0, initOffsets=grid)
    g, o, st = _check(ctx, p, a, b)
    assert (o["type"] == 0).sum() > 50


def test_zero_region_and_edges(ctx, small_pair_np):
    a, b = small_pair_np
    a = a.copy()
    b = b.copy()
    a[:96] = 0
    b[:96] = 0
    p = _p(rStart=0, aStart=0, nR=33, nA=33)
    g, o, st = _check(ctx, p, a, b)
    assert g["stats"]["nAttempted"] == o["stats"]["nAttempted"]


def test_device_resident_inputs(ctx, small_pair_np):
    import torch
    a, b = small_pair_np
    p = _p()
    ta = torch.from_numpy(a).cuda()
    tb = torch.from_numpy(b).cuda()
    out = {k: torch.zeros((p.nA, p.nR), dtype=torch.float32, device="cuda") for k in ("offR", "offA", "corr", "azd")}
    out["type"] = torch.zeros((p.nA, p.nR), dtype=torch.uint8, device="cuda")
    ctx.strack(p, ta, tb, out=out)
    g = ctx.strack(p, a, b)
    for k in ("offR", "offA", "corr", "type"):
        assert np.array_equal(out[k].cpu().numpy(), g[k])


@pytest.mark.parametrize("grid_plan", [False, True])
def test_banded_upload_matches_device_inputs(ctx, grid_plan):
    """Host images go up in azimuth bands overlapped with matching; the
    results equal those of the same images already on the device."""
    import torch
    s1, s2 = synth.small_pair(na=2048, nr=4096, seed=7)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)  # 2 x 64 MiB: several bands
    kw = dict(rStart=40, aStart=40, deltaR=64, deltaA=16, nR=62, nA=124)
    if grid_plan:
        grid = {"nr": 64, "na": 64, "r0": 0.0, "a0": 0.0, "deltaR": 64.0, "deltaA": 32.0,
                "dr": np.full((64, 64), 2.0, np.float32), "da": np.full((64, 64), 0.3, np.float32)}
        kw.update(polyShift=0, initOffsets=grid)
    p = _p(**kw)
    g = ctx.strack(p, a, b)
    assert ctx.launch_count() > 4  # band count + scatter + one complex launch per band
    out = {k: torch.zeros((p.nA, p.nR), dtype=torch.float32, device="cuda") for k in ("offR", "offA", "corr", "azd")}
    out["type"] = torch.zeros((p.nA, p.nR), dtype=torch.uint8, device="cuda")
    ctx.strack(p, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), out=out)
    for k in ("offR", "offA", "corr", "azd", "type"):
        assert np.array_equal(out[k].cpu().numpy(), g[k]), k
    assert (g["type"] > 0).mean() > 0.9


def test_interferogram_phase_correction(ctx):
    """phaseCorrectInt on the GPU against the oracle: a 0.6 rad/px range fringe
    that decorrelates the pair is flattened with the interferogram (big-endian
    host copy and little-endian device copy give the same offsets)."""
    import torch
    s1, s2 = synth.make_pair(512, 1024, 12, dr=lambda y, x: 1.3 + 0.3 * torch.sin(x / 150.0),
                             da=lambda y, x: 0.4 + 0 * x, coherence=0.8, ramp=0.6)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    intf = synth.fringe_interferogram(512, 1024, 4, 2, 0.6)
    for W, nrl, nal in ((32, 4, 2), (64, 4, 2)):
        kw = dict(rStart=W + 8, aStart=W + 8, deltaR=W // 2, deltaA=W // 2, nR=(1024 - 2 * W - 16) // (W // 2),
                  nA=(512 - 2 * W - 16) // (W // 2), wR=W, wA=W, wRa=W, wAa=W)
        fi = synth.fringe_interferogram(512, 1024, nrl, nal, 0.6)
        p = abi.TrackParams(**kw, intf=dict(data=fi, nrl=nrl, nal=nal))
        g, o, st = _check(ctx, p, a, b)
        assert (o["type"] == 1).mean() > 0.9 and (g["type"] == 1).mean() > 0.9
        td = torch.from_numpy(np.ascontiguousarray(fi.astype("<i2"))).cuda()
        g2 = ctx.strack(abi.TrackParams(**kw, intf=dict(data=td, nrl=nrl, nal=nal)), a, b)
        assert np.array_equal(g2["offR"], g["offR"]) and np.array_equal(g2["type"], g["type"])
    with pytest.raises(Exception, match="smaller than the window"):
        ctx.strack(abi.TrackParams(rStart=48, aStart=48, deltaR=16, deltaA=16, nR=4, nA=4,
                                   intf=dict(data=intf, nrl=3, nal=3)), a, b)


@pytest.mark.parametrize("kw", [
    dict(),                                                      # complex matches, 2-D fit on the 2x grid
    dict(noComplex=1),                                           # amplitude: shared-memory kernel (Ws 32)
    dict(noComplex=1, wRa=48, wAa=48, rStart=56, aStart=56),     # amplitude: shared-memory kernel (Ws 48)
    dict(noComplex=1, wR=64, wA=64, wRa=64, wAa=64, deltaR=24, deltaA=24, nR=36, nA=16, rStart=64,
         aStart=64),                                             # amplitude: lean shared-memory kernel (Ws 64)
    dict(wR=64, wA=64, wRa=64, wAa=64, deltaR=24, deltaA=24, nR=36, nA=16, rStart=64, aStart=64),
])
def test_gauss_fit_mode(ctx, pair_1k, kw):
    """-gauss (cmpTrackGauss, speckleTrack.c:2205-2303): the 18 x 18 Gaussian
    fit replaces the 8x8 -> 96x96 oversampling in the complex and amplitude
    stages; offsets and match types against the oracle at the usual bar."""
    a, b = pair_1k
    p = _p(gaussFlag=1, **kw)
    g, o, st = _check(ctx, p, a, b)
    assert st["n_match_oracle"] > 300
    d = ctx.strack(_p(**kw), a, b)
    ok = (g["type"] > 0) & (d["type"] > 0)
    moved = (g["offR"][ok] != d["offR"][ok]) | (g["offA"][ok] != d["offA"][ok])
    assert moved.mean() > 0.2  # the fit, not the oversampling, placed the peaks


def test_gauss_fit_moderate_coherence(ctx):
    """-gauss at coherence 0.55: complex fits fail for about half the points
    and both amplitude tries (32 and 64 windows) place the rest.  (The
    Gaussian has no background term, so at coherence 0.25 the fit settles on
    broad, weak peaks and every point fails, in the oracle as on the GPU.)"""
    s1, s2 = synth.make_pair(512, 512, 21, dr=lambda y, x: 1.3 + 0 * x, da=lambda y, x: -0.6 + 0 * y,
                             coherence=0.55)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    p = _p(rStart=72, aStart=72, nR=24, nA=24, deltaR=16, deltaA=16, gaussFlag=1)
    g, o, st = _check(ctx, p, a, b)
    assert o["stats"]["nAmp"] > 20 and o["stats"]["nAmpL"] > 100 and o["stats"]["nComplex"] > 100


def _baseline_tables(nr, ramp, lam=0.0555):
    """Per-range-sample tables of initPhaseCorrect (speckleTrack.c:1556-1625)
    chosen so that phaseCorrectBaseline's dominant term, -bn sinThetaD ptod,
    is a range ramp of `ramp` rad/px for bn = 1; the cosThetaD and overRange
    terms add small, slowly varying phases so that every term is exercised."""
    ptod = -(4.0 * np.pi) / lam
    j = np.arange(nr, dtype=np.float64)
    sin_t = -ramp * j / ptod + 1e-4 * np.sin(j / 50.0)
    cos_t = 0.9 + 1e-6 * j
    over_r = 1.0 / (850e3 + 2.33 * j)
    return sin_t, cos_t, over_r


def test_baseline_phase_flattening(ctx):
    """phaseCorrectBaseline (speckleTrack.c:868-907) with a non-zero baseline:
    image 2 carries a 0.6 rad/px range fringe that decorrelates the pair; the
    baseline terms (Bn, Bp, dBn, dBp, dBnQ, dBpQ all non-zero) put the same
    fringe on patch 1, so complex matching recovers.  GPU against the oracle
    at the usual bar, at W = 32 and 64."""
    import torch
    s1, s2 = synth.make_pair(512, 1024, 12, dr=lambda y, x: 1.3 + 0.3 * torch.sin(x / 150.0),
                             da=lambda y, x: 0.4 + 0 * x, coherence=0.8, ramp=0.6)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    sin_t, cos_t, over_r = _baseline_tables(1024, 0.6)
    base = dict(Bn=1.0, Bp=2.0, dBn=0.02, dBp=0.3, dBnQ=0.01, dBpQ=0.05, lambda_=0.0555,
                sinThetaD=sin_t, cosThetaD=cos_t, overRange=over_r)
    for W in (32, 64):
        kw = dict(rStart=W + 8, aStart=W + 8, deltaR=W // 2, deltaA=W // 2, nR=(1024 - 2 * W - 16) // (W // 2),
                  nA=(512 - 2 * W - 16) // (W // 2), wR=W, wA=W, wRa=W, wAa=W)
        p = abi.TrackParams(**kw, baseline=base)
        g, o, st = _check(ctx, p, a, b)
        assert (o["type"] == 1).mean() > 0.9 and (g["type"] == 1).mean() > 0.9
        plain = oracle.strack(abi.TrackParams(**kw), a, b)
        assert (plain["type"] == 1).mean() < 0.3  # without the baseline the fringe decorrelates the pair
