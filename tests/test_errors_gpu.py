"""Argument checks of the C ABI on the GPU: every invalid call returns its
error code and a one-line reason before any kernel runs, and the context
stays usable afterwards (the reference exits the process on such input)."""
import numpy as np
import pytest

from specklesource_b200 import abi

pytestmark = pytest.mark.gpu

SB_ERR_ARG, SB_ERR_UNSUPPORTED = abi.SB_ERR_ARG, abi.SB_ERR_UNSUPPORTED


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
    rng = np.random.default_rng(0)
    a = (rng.standard_normal((256, 256)) + 1j * rng.standard_normal((256, 256))).astype(np.complex64)
    return a, np.roll(a, (1, 2), axis=(0, 1))


def _p(**kw):
    base = dict(rStart=64, aStart=64, deltaR=32, deltaA=32, nR=3, nA=3, wR=32, wA=32, wRa=32, wAa=32)
    base.update(kw)
    return abi.TrackParams(**base)


def _fails(fn, code, text):
    from specklesource_b200.runtime import SpeckleError
    with pytest.raises(SpeckleError, match=text) as ei:
        fn()
    assert ei.value.code == code


@pytest.mark.parametrize("kw,code,text", [
    (dict(nR=0), SB_ERR_ARG, "empty grid"),
    (dict(scaleFactor=0), SB_ERR_ARG, "scaleFactor"),
    (dict(polyShift=0), SB_ERR_ARG, "initOffsets"),
    (dict(wR=32, wA=48, wRa=32, wAa=32), SB_ERR_UNSUPPORTED, "square"),
    (dict(wR=40, wA=40, wRa=40, wAa=40), SB_ERR_UNSUPPORTED, "not supported"),
    (dict(wRa=256, wAa=256), SB_ERR_UNSUPPORTED, "amplitude window"),
])
def test_strack_rejects(ctx, pair, kw, code, text):
    a, b = pair
    _fails(lambda: ctx.strack(_p(**kw), a, b), code, text)


def test_strack_rejects_mixed_sample_types(ctx, pair):
    a, _ = pair
    b16 = np.zeros((256, 256, 2), np.int16)
    _fails(lambda: ctx.strack(_p(), a, b16), SB_ERR_ARG, "sample type")


def test_strackw_rejects(ctx, pair):
    a, b = pair
    sw = dict(wRa=64, wAa=64, edgePadR=8, edgePadA=8, navgR=2, navgA=2)
    _fails(lambda: ctx.strackw(_p(**dict(sw, wRa=40, wAa=40)), a, b), SB_ERR_UNSUPPORTED, "search window")
    _fails(lambda: ctx.strackw(_p(**dict(sw, edgePadR=8, edgePadA=4)), a, b), SB_ERR_UNSUPPORTED, "edgeR")
    _fails(lambda: ctx.strackw(_p(**dict(sw, edgePadR=40, edgePadA=40)), a, b), SB_ERR_ARG, "no chip")


def test_cull_rejects(ctx):
    g = np.zeros((20, 30), np.float32)
    mt = np.ones((20, 30), np.uint8)
    _fails(lambda: ctx.cull(abi.CullParams(nR=30, nA=20, bR=40, bA=40), g, g, g, mt), SB_ERR_UNSUPPORTED,
           "32 x 32")
    _fails(lambda: ctx.cull(abi.CullParams(nR=30, nA=20, useSim=1), g, g, g, mt), SB_ERR_ARG, "useSim")
    p = abi.CullLSParams(nx=30, ny=20, deltaT=16.0, dx=15.0, dy=15.0)  # nOver not given
    _fails(lambda: ctx.cullls(p, g, g, mt), SB_ERR_ARG, "nOver")


def test_context_still_works_after_the_errors(ctx, pair):
    a, b = pair
    r = ctx.strack(_p(), a, b)
    assert (r["type"] == abi.SB_CMATCH).all()
    assert np.allclose(r["offR"], 2.0, atol=1 / 24) and np.allclose(r["offA"], 1.0, atol=1 / 24)
