"""strackw on the GPU (through the C ABI) against the FP64 oracle."""
import ctypes as C

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
def shear():
    s1, s2 = synth.shear_pair(device="cpu", na=768, nr=1024, seed=3)
    return synth.to_numpy(s1), synth.to_numpy(s2)


def _p(W, pad, navg, n=(6, 8), step=48, start=None, **kw):
    start = start if start is not None else W // 2 + 8
    base = dict(rStart=start, aStart=start, deltaR=step, deltaA=step, nR=n[1], nA=n[0], wR=W, wA=W, wRa=W, wAa=W,
                edgePadR=pad, edgePadA=pad, navgR=navg, navgA=navg)
    base.update(kw)
    return abi.TrackParams(**base)


def _check(ctx, p, a, b):
    g = ctx.strackw(p, a, b)
    o = oracle.strackw(p, a, b)
    st = compare_track(g, o)
    print(st, g["stats"], o["stats"])
    assert st["pass"], st
    rel = np.abs(g["corr"] - o["corr"]) / np.maximum(1e-6, np.abs(o["corr"]))
    assert np.percentile(rel[o["type"] > 0], 99) < 1e-3
    return g, o


@pytest.mark.parametrize("W,pad,navg,n,step", [(64, 8, 1, (16, 24), 28), (64, 8, 2, (16, 24), 28),
                                                (128, 16, 2, (14, 18), 28), (96, 12, 2, (14, 20), 30),
                                                (192, 32, 2, (5, 7), 48)])
def test_strackw_matches_oracle(ctx, shear, W, pad, navg, n, step):
    a, b = shear
    _check(ctx, _p(W, pad, navg, n=n, step=step), a, b)


def test_strackw_config3_geometry(ctx, shear):
    """Search window 224 (128 + 2 x 48), edge pad 48, 5 x 5 box pre-smoothing."""
    a, b = shear
    p = _p(224, 48, 2, n=(3, 4), step=160, start=120)
    g, o = _check(ctx, p, a, b)
    assert (o["type"] == abi.SB_AMPMATCH).sum() == 12


def test_strackw_int16_msb_and_mask(ctx, shear):
    a, b = shear
    ai = np.stack([np.round(a.real * 2000), np.round(a.imag * 2000)], -1).astype(">i2")
    bi = np.stack([np.round(b.real * 2000), np.round(b.imag * 2000)], -1).astype(">i2")
    mask = np.ones((12, 16), np.uint8)
    mask[::3, ::2] = 0
    p = _p(64, 8, 2, mask={"r0": 0, "a0": 0, "nr": 16, "na": 12, "nrl": 64, "nal": 64, "mask": mask})
    _check(ctx, p, ai, bi)


def test_strackw_offset_grid(ctx, shear):
    a, b = shear
    grid = {"nr": 12, "na": 10, "r0": 0.0, "a0": 0.0, "deltaR": 96.0, "deltaA": 96.0,
            "dr": np.full((10, 12), 3.0, np.float32), "da": np.full((10, 12), -1.0, np.float32)}
    grid["dr"][2:4, 2:4] = -2e9
    p = _p(64, 8, 1, polyShift=0, initOffsets=grid)
    _check(ctx, p, a, b)


def test_est_dop_carrier_batch(ctx):
    import torch
    rng = np.random.default_rng(4)
    nAz, nRg, n = 32, 24, 7
    y = np.arange(nAz)[:, None]
    P1 = np.stack([np.exp(2j * np.pi * f * y) * (1 + 0.1 * rng.standard_normal((nAz, nRg)))
                   for f in np.linspace(-0.3, 0.3, n)]).astype(np.complex64)
    P2 = (P1 * np.exp(1j * rng.uniform(0, 1, (n, 1, 1)))).astype(np.complex64)
    t1 = torch.from_numpy(P1).cuda()
    t2 = torch.from_numpy(P2).cuda()
    out = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc = ctx.lib.sb_est_dop_carrier(ctx.h, t1.data_ptr(), t2.data_ptr(), n, nAz, nRg, nAz, out.data_ptr())
    assert rc == abi.SB_OK
    want = [oracle.est_dop_carrier(P1[k], P2[k], nAz) for k in range(n)]
    assert out.cpu().numpy().tolist() == want


def test_strackw_config3_geometry_240_points():
    """The benchmark's fast-flow geometry (search window 224 = 128 + 2 x 48,
    edge pad 48, 5 x 5 box pre-smoothing) on 240 points spread over a
    2000 x 4000 pair of the shear-zone generator (|d| up to 40 px, coherence
    0.25-0.5), against the FP64 oracle."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from specklesource_b200 import build, runtime
    build.build()
    s1, s2 = synth.shear_pair(device="cuda", na=2000, nr=4000, seed=3)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    del s1, s2
    p = abi.TrackParams(rStart=160, aStart=160, deltaR=160, deltaA=140, nR=20, nA=12, wR=224, wA=224, wRa=224,
                        wAa=224, edgePadR=48, edgePadA=48, navgR=2, navgA=2)
    with runtime.Context(0) as c:
        g, o = _check(c, p, a, b)
    assert (o["type"] == abi.SB_AMPMATCH).sum() >= 200
