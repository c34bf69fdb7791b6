"""cullst on the GPU (through the C ABI) against the oracle: keep masks and
culled offsets bit-exact, smoothed offsets and sigmas within float tolerance."""
import numpy as np
import pytest

from oracle import oracle
from specklesource_b200 import abi
from specklesource_b200.synth import offsets_field

pytestmark = pytest.mark.gpu

LARGE = np.float32(-2e9)


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


def _same(a, b):
    return np.array_equal(a, b, equal_nan=True)


def _check(g, o, keys_exact=("offR", "offA", "type")):
    for k in keys_exact:
        assert _same(g[k], o[k]), f"{k} differs at {np.argwhere(~((g[k] == o[k]) | (np.isnan(g[k]) & np.isnan(o[k]))))[:5]}"
    for k in ("offRS", "offAS"):
        vg, vo = g[k] > -1.9e9, o[k] > -1.9e9
        assert np.array_equal(vg, vo), f"{k} keep mask differs"
        assert np.allclose(g[k][vo], o[k][vo], rtol=1e-6, atol=1e-6)
    for k in ("sigmaR", "sigmaA"):
        vg, vo = g[k] > -1.9e9, o[k] > -1.9e9
        assert np.array_equal(vg, vo), f"{k} validity differs"
        assert np.allclose(g[k][vo], o[k][vo], rtol=2e-3, atol=1e-5)


@pytest.mark.parametrize("kw", [
    dict(),                                                          # cullst defaults
    dict(bR=5, bA=5, nGood=12, sR=3, sA=3, islandThresh=10),          # 5x5 median, 3x3 smoothing, islands
    dict(bR=7, bA=3, nGood=5, maxA=0.5, maxR=0.5, sR=4, sA=1, corrThresh=0.2, islandThresh=4, connectivity=4),
    dict(bR=13, bA=13, nGood=40, islandThresh=6),  # box above 128 values: the row-wavefront median kernel
])
def test_cull_pipeline_matches_oracle(ctx, kw):
    nA, nR = 150, 230
    offR, offA, corr, mt = offsets_field(nA, nR, 7)
    p = abi.CullParams(nR=nR, nA=nA, **kw)
    g = ctx.cull(p, offR, offA, corr, mt)
    o = oracle.cull(p, offR, offA, corr, mt)
    _check(g, o)
    assert g["nCulled"] == o["nCulled"]
    if p.islandThresh > 0:
        assert (g["nIslands"], g["nIslandPoints"]) == (o["nIslands"], o["nIslandPoints"])


def test_cull_single_passes(ctx):
    nA, nR = 80, 120
    offR, offA, corr, mt = offsets_field(nA, nR, 8)
    p = abi.CullParams(nR=nR, nA=nA)
    g = ctx.cull(p, offR, offA, corr, mt, passes=("st",))
    o = oracle.cull(p, offR, offA, corr, mt, passes=("st",))
    assert _same(g["offR"], o["offR"]) and _same(g["offA"], o["offA"])
    g = ctx.cull(p, offR, offA, corr, mt, passes=("st", "stats", "smooth", "islands"))
    o = oracle.cull(p, offR, offA, corr, mt, passes=("st", "stats", "smooth", "islands"))
    _check(g, o)


def test_cull_mask_single_mt_and_sim(ctx):
    nA, nR = 90, 140
    offR, offA, corr, mt = offsets_field(nA, nR, 9)
    rng = np.random.default_rng(3)
    mask = rng.integers(0, 8, (nA, nR)).astype(np.uint8)
    simR = (0.5 * rng.standard_normal((nA, nR))).astype(np.float32)
    simA = (0.5 * rng.standard_normal((nA, nR))).astype(np.float32)
    p = abi.CullParams(nR=nR, nA=nA, singleMT=2, useSim=1, islandThresh=6)
    g = ctx.cull(p, offR, offA, corr, mt, mask=mask, simR=simR, simA=simA)
    o = oracle.cull(p, offR, offA, corr, mt, mask=mask, simR=simR, simA=simA)
    _check(g, o)


def test_cull_large_grid_keep_mask(ctx):
    """Keep masks on a 700 x 993 grid (rows of the large strack workload's grid)."""
    nA, nR = 700, 993
    offR, offA, corr, mt = offsets_field(nA, nR, 10)
    p = abi.CullParams(nR=nR, nA=nA, bR=5, bA=5, nGood=12, sR=3, sA=3, islandThresh=10, nCullPasses=3)
    g = ctx.cull(p, offR, offA, corr, mt)
    t = ctx.timing()
    o = oracle.cull(p, offR, offA, corr, mt)
    _check(g, o)
    print("cull 700x993:", t)
    assert o["nIslands"] > 0


# ---------------------------------------------------------------- cullls

SLOW, NODATA_BIT = 0x10, 0x40  # stand-ins for lstrack.h's SLOWVEL / NODATATOUSE


def _ls_inputs(nA, nR, seed):
    X, Y, _, mt = offsets_field(nA, nR, seed)
    rng = np.random.default_rng(seed + 100)
    yy, xx = np.mgrid[0:nA, 0:nR]
    t = np.where((xx - nR / 3) ** 2 + (yy - nA / 2) ** 2 < (nA / 3) ** 2, SLOW, 0)  # a slow-moving disc
    t = t | np.where(rng.random((nA, nR)) < 0.05, NODATA_BIT, 0) | (mt & 3)
    return X, Y, t.astype(np.uint8)


def _check_ls(g, o):
    for k in ("X", "Y"):
        assert _same(g[k], o[k]), f"{k} differs at {np.argwhere(~((g[k] == o[k]) | (np.isnan(g[k]) & np.isnan(o[k]))))[:5]}"
    for k in ("XS", "YS"):
        vg, vo = g[k] > -1.9e9, o[k] > -1.9e9
        assert np.array_equal(vg, vo), f"{k} keep mask differs"
        assert np.allclose(g[k][vo], o[k][vo], rtol=1e-6, atol=1e-6)
    for k in ("sigmaX", "sigmaY"):
        vg, vo = g[k] > -1.9e9, o[k] > -1.9e9
        assert np.array_equal(vg, vo), f"{k} validity differs"
        assert np.allclose(g[k][vo], o[k][vo], rtol=2e-3, atol=1e-5)
    for k in ("nAttempt", "nMatch", "nCulled", "nIslands", "nIslandPoints"):
        assert g[k] == o[k], k


@pytest.mark.parametrize("kw", [
    dict(islandThresh=6),                                                   # cullls defaults, islands
    dict(boxSize=5, nGood=8, sX=1, sY=5, noDataLimit=-3.0, connectivity=4, islandThresh=3),
    dict(boxSize=13, nGood=40, deltaT=24.0, dx=30.0, dy=30.0),              # box above 128 values: the wavefront kernel
])
def test_cullls_matches_oracle(ctx, kw):
    nA, nR = 150, 230
    X, Y, t = _ls_inputs(nA, nR, 11)
    base = dict(nx=nR, ny=nA, deltaT=365.0, dx=15.0, dy=15.0, nOver=10.0, slowVelMask=SLOW, noDataMask=NODATA_BIT)
    base.update(kw)
    p = abi.CullLSParams(**base)
    g = ctx.cullls(p, X, Y, t)
    o = oracle.cullls(p, X, Y, t)
    _check_ls(g, o)
    assert o["nCulled"] > 0 and o["nMatch"] > o["nCulled"]


def test_cullls_large_grid(ctx):
    nA, nR = 700, 993
    X, Y, t = _ls_inputs(nA, nR, 12)
    p = abi.CullLSParams(nx=nR, ny=nA, deltaT=48.0, dx=15.0, dy=15.0, nOver=10.0, slowVelMask=SLOW,
                         noDataMask=NODATA_BIT, islandThresh=10)
    g = ctx.cullls(p, X, Y, t)
    o = oracle.cullls(p, X, Y, t)
    _check_ls(g, o)
    assert o["nIslands"] > 0


def test_wavefront_wait_times_out_and_context_stays_usable(ctx):
    """The row-wavefront median kernel (13 x 13 box) waits for the previous
    grid row with a bounded wait.  With a limit of 0 naps the first unmet
    check gives up: the call fails with SB_ERR_TIMEOUT (nothing hangs), and the
    same context then culls the grid bit-exactly with the default limit."""
    from specklesource_b200.runtime import SpeckleError
    nA, nR = 150, 230
    offR, offA, corr, mt = offsets_field(nA, nR, 7)
    p = abi.CullParams(nR=nR, nA=nA, bR=13, bA=13, nGood=40, islandThresh=6)
    assert ctx.lib.sb_set_wait_limit(ctx.h, -1) == abi.SB_ERR_ARG
    assert ctx.lib.sb_set_wait_limit(ctx.h, 0) == abi.SB_OK
    try:
        with pytest.raises(SpeckleError, match="timed out") as ei:
            ctx.cull(p, offR, offA, corr, mt)
        assert ei.value.code == abi.SB_ERR_TIMEOUT
    finally:
        assert ctx.lib.sb_set_wait_limit(ctx.h, 1 << 26) == abi.SB_OK
    g = ctx.cull(p, offR, offA, corr, mt)
    o = oracle.cull(p, offR, offA, corr, mt)
    _check(g, o)
    assert g["nCulled"] == o["nCulled"]
