"""Known-answer tests of the CPU oracle (the reference ships none).

Beside the comparison with the reference's own code (tests/test_ref_pin.py),
these tests pin the oracle to properties the reference's algorithm must have:
FFTW-convention transforms, exact recovery of integer and band-limited
sub-pixel shifts, in-band failure values, and the cull rules on hand-built
grids.
"""
import numpy as np
import pytest

from oracle import oracle
from specklesource_b200 import abi, synth

LARGE = float(abi.SB_LARGEINT)


def _speckle(na, nr, seed, band=0.8):
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((na, nr)) + 1j * rng.standard_normal((na, nr))
    Z = np.fft.fft2(z)
    fy = np.abs(np.fft.fftfreq(na)) <= band / 2
    fx = np.abs(np.fft.fftfreq(nr)) <= band / 2
    z = np.fft.ifft2(Z * (fy[:, None] & fx[None, :]))
    return z / np.sqrt(np.mean(np.abs(z) ** 2))


def _fourier_shift(z, da, dr):
    """z2(y, x) = z(y - da, x - dr) exactly (periodic, band-limited)."""
    na, nr = z.shape
    fy = np.fft.fftfreq(na)[:, None]
    fx = np.fft.fftfreq(nr)[None, :]
    return np.fft.ifft2(np.fft.fft2(z) * np.exp(-2j * np.pi * (fy * da + fx * dr)))


@pytest.mark.parametrize("shape,sign", [((8, 8), -1), ((24, 32), -1), ((96, 96), 1), ((21, 21), 1), ((28, 14), -1)])
def test_fft_matches_numpy_convention(shape, sign):
    rng = np.random.default_rng(0)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    got = oracle.fft2d(x, sign)
    want = np.fft.fft2(x) if sign < 0 else np.fft.ifft2(x) * x.size
    assert np.allclose(got, want, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("shape", [(8, 8), (24, 32), (21, 21), (28, 14), (35, 10), (96, 96), (224, 112), (448, 64)])
def test_batched_float_fft_matches_numpy(shape):
    """The float library's vectorised 2-D FFT (self-sorting, radix 4/2/3/7 and
    the direct sum for other factors), both signs, to float accuracy."""
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    for sign in (-1, 1):
        got = oracle.fft2d(x, sign, precision="f32")
        want = np.fft.fft2(x) if sign < 0 else np.fft.ifft2(x) * x.size
        assert np.abs(got - want).max() <= 2e-6 * np.abs(want).max()


def _params(**kw):
    base = dict(rStart=48, aStart=48, deltaR=16, deltaA=16, nR=10, nA=10, wR=32, wA=32, wRa=32, wAa=32)
    base.update(kw)
    return abi.TrackParams(**base)


@pytest.mark.parametrize("dr,da", [(3, -2), (-5, 4), (0, 0)])
def test_integer_shift_is_recovered(dr, da):
    z = _speckle(256, 256, 11)
    z2 = np.roll(z, (da, dr), axis=(0, 1))
    p = _params()
    o = oracle.strack(p, z.astype(np.complex64), z2.astype(np.complex64))
    assert (o["type"] == abi.SB_CMATCH).all()
    # offsets are multiples of the 1/24 px quantum; an exact shift lands within one
    assert np.abs(o["offR"] - dr).max() <= 1 / 24 + 1e-6
    assert np.abs(o["offA"] - da).max() <= 1 / 24 + 1e-6
    assert (o["corr"] > 0.9).all()


@pytest.mark.parametrize("dr,da", [(1.25, -0.5), (-2.4, 0.3), (0.7, 1.9)])
def test_subpixel_shift_within_quantum(dr, da):
    z = _speckle(256, 256, 12)
    z2 = _fourier_shift(z, da, dr)
    p = _params()
    o = oracle.strack(p, z.astype(np.complex64), z2.astype(np.complex64))
    assert (o["type"] == abi.SB_CMATCH).all()
    assert np.median(np.abs(o["offR"] - dr)) <= 1 / 24
    assert np.median(np.abs(o["offA"] - da)) <= 1 / 24
    assert np.abs(o["offR"] - dr).max() <= 2 / 24


def test_amplitude_only_tracks_shift():
    z = _speckle(256, 256, 13)
    z2 = _fourier_shift(z, 0.5, 2.25)
    p = _params(noComplex=1)
    o = oracle.strack(p, z.astype(np.complex64), z2.astype(np.complex64))
    assert (o["type"] == abi.SB_AMPMATCH).all()
    assert np.median(np.abs(o["offR"] - 2.25)) < 0.1
    assert np.median(np.abs(o["offA"] - 0.5)) < 0.1


def test_zero_patch_fails_in_band():
    z = _speckle(256, 256, 14)
    z2 = z.copy()
    z[:128, :] = 0
    z2[:128, :] = 0
    p = _params()
    o = oracle.strack(p, z.astype(np.complex64), z2.astype(np.complex64))
    top = o["type"][:3]  # grid rows whose windows lie in the zeroed half
    assert (top == abi.SB_BAD).all()
    assert (o["offR"][:3] == -LARGE).all() and (o["offA"][:3] == -LARGE).all()
    assert (o["corr"][:3] == 0).all()
    assert (o["type"][-3:] == abi.SB_CMATCH).all()


def test_out_of_bounds_points_are_bad():
    z = _speckle(128, 128, 15)
    p = _params(rStart=0, aStart=0, nR=3, nA=3)  # first row/col windows start at -16
    o = oracle.strack(p, z.astype(np.complex64), z.astype(np.complex64))
    assert (o["type"][0, :] == abi.SB_BAD).all() and (o["type"][:, 0] == abi.SB_BAD).all()
    assert o["stats"]["nAttempted"] == 9


def test_big_endian_input_is_identical():
    z = _speckle(128, 128, 16).astype(np.complex64)
    z2 = np.roll(z, (1, 2), axis=(0, 1))
    p = _params(rStart=40, aStart=40, nR=4, nA=4)
    a = oracle.strack(p, z, z2)
    b = oracle.strack(p, z.astype(">c8"), z2.astype(">c8"))
    for k in ("offR", "offA", "corr", "type", "azd"):
        assert np.array_equal(a[k], b[k])


def test_f32_oracle_agrees_with_f64(small_pair_np):
    a, b = small_pair_np
    p = _params(rStart=40, aStart=40, nR=28, nA=28, deltaR=16, deltaA=8)
    o64 = oracle.strack(p, a, b, precision="f64")
    o32 = oracle.strack(p, a, b, precision="f32")
    ok = o64["type"] > 0
    assert (o64["type"] == o32["type"]).mean() >= 0.99
    d = np.abs(o64["offR"] - o32["offR"])[ok & (o32["type"] > 0)]
    assert (d <= 0.01).mean() >= 0.99


def test_doppler_roll_of_a_carrier():
    # a pure azimuth carrier exp(2 pi i f y) gives roll round(nAz/2 * 2 f)
    na = nr = 32
    y = np.arange(na)[:, None] * np.ones((1, nr))
    rng = np.random.default_rng(3)
    for f in (0.05, 0.2, -0.15):
        z = np.exp(2j * np.pi * f * y) * (1 + 0.01 * rng.standard_normal((na, nr)))
        s = oracle.est_dop_carrier(z, z, na)
        want = int(np.floor(na / 2 * 2 * f + 0.5)) if f >= 0 else int(np.ceil(na / 2 * 2 * f - 0.5))
        if want < 0:
            want += na
        assert s == want


# ---------------------------------------------------------------- cull


def _grid(nA=30, nR=40, seed=0):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:nA, 0:nR]
    offR = (0.5 + 0.01 * xx + 0.005 * yy + 0.02 * rng.standard_normal((nA, nR))).astype(np.float32)
    offA = (-0.3 + 0.004 * xx + 0.02 * rng.standard_normal((nA, nR))).astype(np.float32)
    corr = np.full((nA, nR), 0.5, np.float32)
    mt = np.ones((nA, nR), np.uint8)
    return offR, offA, corr, mt


def test_cull_removes_isolated_outlier():
    offR, offA, corr, mt = _grid()
    offR[10, 10] += 5.0
    p = abi.CullParams(nR=40, nA=30, islandThresh=-1)
    d = oracle.cull(p, offR, offA, corr, mt, passes=("st",))
    assert d["offR"][10, 10] == -LARGE
    assert (d["offR"][12:20, 12:20] > -LARGE).all()


def test_cull_needs_enough_neighbours():
    offR, offA, corr, mt = _grid()
    p = abi.CullParams(nR=40, nA=30, nGood=17)
    d = oracle.cull(p, offR, offA, corr, mt, passes=("st",))
    # a 9x9 box clipped at a corner holds 25 points (> 17): kept
    assert d["offR"][0, 0] > -LARGE
    p = abi.CullParams(nR=40, nA=30, nGood=30)
    d = oracle.cull(p, offR, offA, corr, mt, passes=("st",))
    assert d["offR"][0, 0] == -LARGE and d["offR"][15, 20] > -LARGE


def test_cull_corr_threshold():
    offR, offA, corr, mt = _grid()
    corr[5, 5] = 0.05
    p = abi.CullParams(nR=40, nA=30, corrThresh=0.1)
    d = oracle.cull(p, offR, offA, corr, mt, passes=("st",))
    assert d["offR"][5, 5] == -LARGE and d["type"][5, 5] == 0


def test_cull_nan_survives_median_pass_then_dropped():
    offR, offA, corr, mt = _grid()
    offR[15, 15] = np.nan
    p = abi.CullParams(nR=40, nA=30)
    d = oracle.cull(p, offR, offA, corr, mt, passes=("st",))
    assert np.isnan(d["offR"][15, 15])
    d = oracle.cull(p, offR, offA, corr, mt)
    assert d["offRS"][15, 15] == -LARGE
    assert d["sigmaA"][15, 15] == -LARGE


def test_cull_smoothing_weights():
    nA, nR = 20, 20
    offR = np.zeros((nA, nR), np.float32)
    offR[:, 10] = 1.0  # a column of ones
    offA = np.zeros((nA, nR), np.float32)
    corr = np.ones((nA, nR), np.float32)
    mt = np.ones((nA, nR), np.uint8)
    p = abi.CullParams(nR=nR, nA=nA, sR=2, sA=1, nGood=0, maxA=10, maxR=10)
    d = oracle.cull(p, offR, offA, corr, mt, passes=("stats", "smooth"))
    # weights 0.5, 1, 0.5 across range: neighbours of the column see 0.5/2
    assert d["offRS"][10, 10] == pytest.approx(1.0 / 2.0)
    assert d["offRS"][10, 9] == pytest.approx(0.5 / 2.0)


def test_cull_islands_by_extent_and_last_label():
    nA, nR = 30, 30
    offRS = np.full((nA, nR), -LARGE, np.float32)
    offRS[2:5, 2:5] = 1.0      # island A, extent 2 (first label)
    offRS[10:25, 10:25] = 1.0  # big region, extent 14
    offRS[27:29, 27:29] = 1.0  # island C, extent 1 (last label: never culled)
    d = {"offRS": offRS}
    p = abi.CullParams(nR=nR, nA=nA, islandThresh=5)
    r = oracle.cull(p, offRS.copy(), offRS.copy(), np.ones((nA, nR)), np.ones((nA, nR), np.uint8),
                    passes=())
    r["offRS"][:] = offRS
    r["offAS"][:] = offRS
    from oracle.oracle import _cull_data, lib
    import ctypes as C
    dd, cd = _cull_data(offRS, offRS, np.ones((nA, nR)), np.ones((nA, nR)))
    dd["offRS"][:] = offRS
    dd["offAS"][:] = offRS
    cp = p.to_c()
    lib("f64").oracle_cull_islands(C.byref(cp), C.byref(cd))
    out = dd["offRS"]
    assert (out[2:5, 2:5] == -LARGE).all()
    assert (out[10:25, 10:25] == 1.0).all()
    assert (out[27:29, 27:29] == 1.0).all()
    assert cd.nIslands == 1
    del d, r


def test_interferogram_flattening_restores_matches():
    """phaseCorrectInt: a 0.6 rad/px range fringe between the images shifts
    their spectra apart and destroys the complex correlation; with the
    interferogram describing it, every point matches at the true offsets."""
    s1, s2 = synth.make_pair(256, 512, 11, dr=lambda y, x: 1.3 + 0 * x, da=lambda y, x: 0.4 + 0 * x,
                             coherence=0.8, ramp=0.6)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    intf = synth.fringe_interferogram(256, 512, 4, 2, 0.6)
    base = dict(rStart=40, aStart=40, deltaR=16, deltaA=16, nR=27, nA=12, wR=32, wA=32, wRa=32, wAa=32, maxTries=0)
    plain = oracle.strack(abi.TrackParams(**base), a, b)
    flat = oracle.strack(abi.TrackParams(**base, intf=dict(data=intf, nrl=4, nal=2)), a, b)
    assert (plain["type"] == 1).mean() < 0.1
    m = flat["type"] == 1
    assert m.all()
    assert abs(np.median(flat["offR"][m]) - 1.3) < 0.05 and abs(np.median(flat["offA"][m]) - 0.4) < 0.05
    # a little-endian copy of the same interferogram gives the same result
    flat2 = oracle.strack(abi.TrackParams(**base, intf=dict(data=intf.astype("<i2"), nrl=4, nal=2)), a, b)
    assert np.array_equal(flat["offR"], flat2["offR"])
    # looks that make the padded patch smaller than the window are refused
    with pytest.raises(RuntimeError):
        oracle.strack(abi.TrackParams(**base, intf=dict(data=intf, nrl=3, nal=3)), a, b)


@pytest.mark.parametrize("dr,da", [(3, -2), (1.25, -0.5), (-2.4, 0.3)])
def test_gauss_fit_recovers_shift(dr, da):
    """-gauss (cmpTrackGauss): the 18 x 18 Gaussian fit places band-limited
    shifts within the 1/24 px quantum in the complex stage and within 1/8 px
    in the amplitude stage; the float oracle gives the same offsets."""
    z = _speckle(256, 256, 12)
    z2 = _fourier_shift(z, da, dr)
    for nc, tol in ((0, 1 / 24), (1, 1 / 8)):
        p = _params(gaussFlag=1, noComplex=nc)
        o = oracle.strack(p, z.astype(np.complex64), z2.astype(np.complex64))
        assert (o["type"] == (abi.SB_AMPMATCH if nc else abi.SB_CMATCH)).all()
        assert np.abs(o["offR"] - dr).max() <= tol + 1e-6
        assert np.abs(o["offA"] - da).max() <= tol + 1e-6
        assert (o["corr"] <= 1.0).all() and (o["corr"] > 0.185).all()
        f = oracle.strack(p, z.astype(np.complex64), z2.astype(np.complex64), precision="f32")
        assert np.array_equal(f["offR"], o["offR"]) and np.array_equal(f["offA"], o["offA"])



# ---------------------------------------------------------------- cullls

SLOW, NODATA_BIT = 0x10, 0x40  # stand-ins for lstrack.h's SLOWVEL / NODATATOUSE


def _ls_params(**kw):
    base = dict(nx=40, ny=30, deltaT=365.0, dx=15.0, dy=15.0, nOver=10.0, slowVelMask=SLOW,
                noDataMask=NODATA_BIT)
    base.update(kw)
    return abi.CullLSParams(**base)


def test_cullls_slow_flow_limits():
    """cullLSData.c:99-117: where every valid box point is slow-moving the
    limits are 40 m/yr * deltaT / pixel size (here 2.67 px), not maxX/maxY."""
    X, Y, _, _ = _grid()
    X[10, 10] += 1.5
    slow = np.full(X.shape, SLOW, np.uint8)
    d = oracle.cullls(_ls_params(), X, Y, slow)
    assert d["X"][10, 10] > -LARGE  # 1.5 px within the slow limit
    d = oracle.cullls(_ls_params(), X, Y, np.zeros(X.shape, np.uint8))
    assert d["X"][10, 10] == -LARGE  # above maxX = 0.75
    mixed = slow.copy()
    mixed[13, 13] = 0  # one fast point in the 9x9 box: the normal limits
    d = oracle.cullls(_ls_params(), X, Y, mixed)
    assert d["X"][10, 10] == -LARGE
    # a year over 1 km pixels: 0.04 px, floored at 0.2
    X2, Y2, _, _ = _grid()
    X2[10, 10] += 0.3
    assert oracle.cullls(_ls_params(dx=1000.0, dy=1000.0), X2, Y2, slow)["X"][10, 10] == -LARGE
    assert oracle.cullls(_ls_params(dx=1000.0, dy=1000.0), X2, Y2, 0 * slow)["X"][10, 10] > -LARGE


def test_cullls_nodata_gate_and_counts():
    X, Y, _, _ = _grid()
    X[3, 3] = -LARGE
    Y[3, 3] = -LARGE
    mt = np.zeros(X.shape, np.uint8)
    mt[0, :5] = NODATA_BIT
    Y[20, 20] = -1.5  # below the NODATA + 1 limit set next
    d = oracle.cullls(_ls_params(noDataLimit=-1.0, maxY=5.0), X, Y, mt)
    assert d["nMatch"] == 40 * 30 - 1 and d["nAttempt"] == 40 * 30 - 5
    assert d["X"][20, 20] == -LARGE


def test_cullls_stats_quantisation_and_plain_smoothing():
    """On an exact plane the stats see only the 1e-5 floor plus (1/NOVER)^2/12
    (cullLSStats.c:147-148); the smoothing is the unweighted 3x3 mean and
    divides the sigmas by sqrt(9)."""
    ny, nx = 30, 40
    yy, xx = np.mgrid[0:ny, 0:nx]
    X = (0.5 + 0.01 * xx + 0.02 * yy).astype(np.float32)
    Y = (-0.2 + 0.005 * xx).astype(np.float32)
    d = oracle.cullls(_ls_params(nOver=10.0), X, Y, np.zeros((ny, nx), np.uint8))
    s = np.sqrt(np.float32(1e-5) + (0.1 * 0.1) / 12.0) / 3.0
    assert d["sigmaX"][15, 20] == pytest.approx(s, rel=1e-5)
    assert d["sigmaY"][15, 20] == pytest.approx(s, rel=1e-5)
    assert d["XS"][15, 20] == pytest.approx(float(X[14:17, 19:22].astype(np.float64).mean()), rel=1e-6)
    assert d["YS"][0, 0] == pytest.approx(float(Y[0:2, 0:2].astype(np.float64).mean()), rel=1e-6)


def test_cullls_writer(tmp_path):
    """writeLSCulledOffsets: big-endian grids and the .cull.dat summary."""
    from specklesource_b200 import files
    X, Y, _, _ = _grid()
    X[10, 10] += 3.0
    mt = np.full(X.shape, 1, np.uint8)
    mt[0, :4] |= NODATA_BIT
    p = _ls_params()
    d = oracle.cullls(p, X, Y, mt)
    meta = dict(fileEarly="a.tif", fileLate="b.tif", x0=-100000.0, y0=250000.0, dx=15.0, dy=15.0, stepX=16,
                stepY=8, slowFlag=1, proj=3413, jdEarly=2459000.5, jdLate=2459016.5)
    root = str(tmp_path / "match")
    n_good, sx, sy = files.write_ls_culled(root, d, p, meta)
    assert n_good == int(((d["XS"] > -1.9e9) & (d["YS"] > -1.9e9)).sum())
    assert np.array_equal(np.fromfile(root + ".cull.dx", ">f4").reshape(X.shape), d["XS"])
    assert np.array_equal(np.fromfile(root + ".cull.sy", ">f4").reshape(X.shape), d["sigmaY"])
    txt = open(root + ".cull.dat").read().splitlines()
    assert txt[6] == "stepY = 16" and txt[7] == "stepX = 8"
    assert txt[14] == "IntervalBetweenImages =    16"
    assert txt[15] == f"Success_rate_for_attempted_matches(%) =  {100.0 * 1200 / 1196:7.2f} "
    assert txt[-1] == "& "
