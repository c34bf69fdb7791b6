"""The split-BF16 tensor-core form of strack's complex stage (SB_FORM_SPLIT_BF16)
against the FP64 oracle, through the C ABI.

The form replaces the complex stage's 64-point DFTs with DFT-GEMMs on the
tcgen05 tensor cores (operands split into hi + lo bfloat16, three products,
FP32 accumulation); everything after the correlation surface is the FP32
form's.  The bar is the tracking bar of the other GPU tests: on the points the
oracle matches, offsets within 0.01 px (complex) / 0.02 px (amplitude) on at
least 99.5 %, match types identical on at least 99.5 % of all points.  The
per-offset and per-peak-value (corr) errors are printed for the record.
"""
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
    c.set_form(abi.SB_FORM_SPLIT_BF16)
    yield c
    c.close()


@pytest.fixture(scope="module")
def pair_1k():
    s1, s2 = synth.small_pair(na=1024, nr=2048)
    return synth.to_numpy(s1), synth.to_numpy(s2)


def _w64(**kw):
    base = dict(rStart=64, aStart=64, deltaR=24, deltaA=24, nR=40, nA=20, wR=64, wA=64, wRa=64, wAa=64)
    base.update(kw)
    return abi.TrackParams(**base)


def _errors(g, o):
    both = (g["type"] > 0) & (o["type"] > 0)
    e = np.maximum(np.abs(g["offR"].astype(np.float64) - o["offR"]), np.abs(g["offA"].astype(np.float64) - o["offA"]))
    c = np.abs(g["corr"].astype(np.float64) - o["corr"]) / np.maximum(1e-6, np.abs(o["corr"]))
    return {"offset_err_px_p50": float(np.percentile(e[both], 50)), "offset_err_px_max": float(e[both].max()),
            "corr_rel_p50": float(np.percentile(c[both], 50)), "corr_rel_p99": float(np.percentile(c[both], 99))}


def _check(ctx, p, a, b, form=abi.SB_FORM_SPLIT_BF16):
    g = ctx.strack(p, a, b)
    assert ctx.last_form() == form
    o = oracle.strack(p, a, b)
    st = compare_track(g, o)
    print(st, _errors(g, o))
    assert st["pass"], st
    return g, o, st


def test_split_bf16_w64_matches_oracle(ctx, pair_1k):
    a, b = pair_1k
    g, o, st = _check(ctx, _w64(), a, b)
    assert st["n_match_oracle"] > 700
    assert np.percentile(np.abs(g["corr"] - o["corr"])[o["type"] == 1] / o["corr"][o["type"] == 1], 99) < 1e-3


def test_split_bf16_large_pair_generator(ctx):
    """The benchmark's 12000 x 24000 generator (coherence per 512-px block in
    [0.3, 0.9], displacement up to 12 px) on a 2400 x 4800 pair, W = 64, step
    24 x 6: a 14 x 196 block of the grid (2,744 points, amplitude fallbacks
    included)."""
    s1, s2 = synth.large_pair(device="cpu", na=2400, nr=4800)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    p = _w64(rStart=96, aStart=600, deltaR=24, deltaA=6, nR=196, nA=14)
    g, o, st = _check(ctx, p, a, b)
    assert st["n_match_oracle"] > 2000


def test_split_bf16_inputs_and_flags(ctx, pair_1k):
    a, b = pair_1k
    _check(ctx, _w64(hanningFlag=0, maxTries=1), a, b)
    sc = 3000.0
    ai = np.stack([np.round(a.real * sc), np.round(a.imag * sc)], -1).astype(np.int16)
    bi = np.stack([np.round(b.real * sc), np.round(b.imag * sc)], -1).astype(np.int16)
    _check(ctx, _w64(nR=20, nA=10), ai.astype(">i2"), bi.astype(">i2"))
    _check(ctx, _w64(nR=20, nA=10), a.astype(">c8"), b.astype(">c8"))


def test_split_bf16_device_inputs_equal_host_inputs(ctx, pair_1k):
    import torch
    a, b = pair_1k
    p = _w64()
    g = ctx.strack(p, a, b)
    d = ctx.strack(p, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    for k in ("offR", "offA", "corr", "type"):
        assert np.array_equal(g[k], d[k]), k


def test_split_bf16_falls_back_where_unsupported(ctx, pair_1k):
    """-gauss, a window other than 64 and a baseline run the FP32 form."""
    a, b = pair_1k
    _check(ctx, _w64(gaussFlag=1, nR=12, nA=8), a, b, form=abi.SB_FORM_FP32)
    _check(ctx, abi.TrackParams(rStart=40, aStart=40, deltaR=16, deltaA=8, nR=27, nA=25), a, b,
           form=abi.SB_FORM_FP32)
