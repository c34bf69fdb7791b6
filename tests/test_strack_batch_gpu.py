"""Batched strack (sb_strack_batch) against one sb_strack call per pair.

A batch groups its pairs by window size and runs every stage once per group
over all the group's points, with the images of all pairs in two atlases; per
point the arithmetic is sb_strack's, so each pair's grids and statistics must
equal its own sb_strack result bit for bit -- with pairs of different sizes,
windows, grids, initial shifts (polynomial and offset grid with holes), masks,
host and device images, and in both transform forms.
"""
import numpy as np
import pytest

from specklesource_b200 import abi, synth

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


def _pairs():
    rng = np.random.default_rng(9)
    cases = []
    for k, (na, nr, W) in enumerate([(512, 768, 32), (700, 512, 64), (640, 1024, 24), (512, 640, 48),
                                      (896, 700, 64), (600, 800, 32), (520, 900, 48), (768, 768, 24),
                                      (1024, 600, 64), (560, 560, 32)]):
        s1, s2 = synth.small_pair(device="cuda", na=na, nr=nr, seed=60 + k)
        step = max(8, W // 2)
        m = W + 8
        kw = dict(rStart=m, aStart=m, deltaR=step, deltaA=step + 4 * (k % 3), wR=W, wA=W, wRa=W, wAa=W)
        kw["nR"] = (nr - 2 * m) // kw["deltaR"] + 1
        kw["nA"] = (na - 2 * m) // kw["deltaA"] + 1
        if k == 3:  # offset-grid initial shift with holes
            g = {"nr": 12, "na": 10, "r0": 0.0, "a0": 0.0, "deltaR": 64.0, "deltaA": 64.0,
                 "dr": np.full((10, 12), 2.0, np.float32), "da": np.full((10, 12), 0.5, np.float32)}
            g["dr"][2:4, 3:6] = -2e9
            kw.update(polyShift=0, initOffsets=g)
        if k == 5:  # mask
            mk = (rng.random((20, 30)) > 0.25).astype(np.uint8)
            kw["mask"] = {"r0": 0, "a0": 0, "nr": 30, "na": 20, "nrl": 32, "nal": 32, "mask": mk}
        if k == 7:
            kw.update(rShiftPoly=(1.0, 0.001, 0.0), aShiftPoly=(-0.5, 0.0, 0.0005))
        p = abi.TrackParams(**kw)
        # alternate host and device images
        a, b = (s1, s2) if k % 2 else (synth.to_numpy(s1), synth.to_numpy(s2))
        cases.append((p, a, b))
    return cases


@pytest.mark.parametrize("form", [abi.SB_FORM_FP32, abi.SB_FORM_SPLIT_BF16])
def test_batch_equals_single_calls(ctx, form):
    cases = _pairs()
    ctx.set_form(form)
    try:
        single = [ctx.strack(p, a, b) for p, a, b in cases]
        batch = ctx.strack_batch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases])
    finally:
        ctx.set_form(abi.SB_FORM_FP32)
    for k, (s, t) in enumerate(zip(single, batch)):
        for key in ("offR", "offA", "corr", "azd", "type"):
            assert np.array_equal(s[key], t[key], equal_nan=True), (k, key)
        assert s["stats"] == t["stats"], k
        assert (t["type"] > 0).mean() > 0.5, k
    assert ctx.launch_count() < 10 * 14  # stages run per window group, not per pair


def test_batch_rejects_mixed_flags(ctx):
    from specklesource_b200.runtime import SpeckleError
    cases = _pairs()[:2]
    cases[1][0].hanningFlag = 0
    with pytest.raises(SpeckleError, match="same for every pair"):
        ctx.strack_batch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases])


def test_batch_more_buckets_than_partition_keys(ctx):
    """35 (complex, amplitude) window buckets, above the 32 keys of one
    ordered partition: the batch plans every pair on the host and must still
    equal each pair's own call."""
    cases = []
    k = 0
    for W in (16, 24, 32, 48, 64):
        for WA in (16, 24, 32, 48, 64, 96, 128):
            s1, s2 = synth.small_pair(device="cuda", na=400, nr=400, seed=200 + k)
            p = abi.TrackParams(rStart=80, aStart=80, deltaR=24, deltaA=24, nR=11, nA=11, wR=W, wA=W, wRa=WA,
                                wAa=WA, maxTries=1)
            cases.append((p, s1, s2))
            k += 1
    single = [ctx.strack(p, a, b) for p, a, b in cases]
    batch = ctx.strack_batch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases])
    for k, (s, t) in enumerate(zip(single, batch)):
        for key in ("offR", "offA", "corr", "azd", "type"):
            sv = s[key].cpu().numpy() if hasattr(s[key], "cpu") else s[key]
            tv = t[key].cpu().numpy() if hasattr(t[key], "cpu") else t[key]
            assert np.array_equal(sv, tv, equal_nan=True), (k, key)
        assert s["stats"] == t["stats"], k
