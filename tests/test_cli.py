"""The drop-in command lines (strack, strackw, cullst).

CPU: argument and parameter-file handling up to the point where a GPU is
needed.  GPU: whole runs on files, outputs compared bit for bit with the
library called directly, and the .dat/.vrt sidecars checked.
"""
import os
import subprocess

import numpy as np
import pytest

from specklesource_b200 import abi, build, files, synth

BIN = os.path.join(os.path.dirname(build.__file__), "bin")


@pytest.fixture(scope="module")
def tools():
    build.build()
    return {n: os.path.join(BIN, n) for n in ("strack", "strackw", "cullst")}


def _run(exe, args, cwd):
    return subprocess.run([exe] + args, cwd=cwd, capture_output=True, text=True, timeout=600)


@pytest.fixture(scope="module")
def pair():
    s1, s2 = synth.small_pair(na=256, nr=512)
    return synth.to_numpy(s1), synth.to_numpy(s2)


def _setup_track(tmp, a, b, **over):
    files.write_slc(str(tmp / "img1.slc"), a)
    files.write_slc(str(tmp / "img2.slc"), b)
    files.write_poly(str(tmp / "offsets.poly"))
    kv = dict(image1="img1.slc", image2="img2.slc", outputfile="out", initialoffsetfile="offsets.poly",
              intgeodat="dummy.geodat", rstart=40, astart=40, deltar=16, deltaa=8, nR=27, nA=25, wr=32, wa=32,
              wra=32, waa=32, navgR=1, navgA=1)
    kv.update(over)
    files.write_parfile(str(tmp / "track.par"), **kv)
    return kv


def test_usage_and_bad_flags(tools, tmp_path):
    for exe in tools.values():
        r = _run(exe, [], tmp_path)
        assert r.returncode == 1 and "parFile" in r.stderr or "inbase" in r.stderr
    r = _run(tools["strack"], ["-bogus", "x.par"], tmp_path)
    assert r.returncode == 1


def test_missing_keys_are_reported(tools, tmp_path, pair):
    a, b = pair
    _setup_track(tmp_path, a, b)
    txt = (tmp_path / "track.par").read_text().replace("navgR", "navgX")
    (tmp_path / "track.par").write_text(txt)
    r = _run(tools["strack"], ["track.par"], tmp_path)
    assert r.returncode == 1 and "navgR not specified" in r.stderr


def test_par_image_descriptions_refused(tools, tmp_path, pair):
    a, b = pair
    _setup_track(tmp_path, a, b)
    os.remove(tmp_path / "img1.slc.vrt")
    with open(tmp_path / "track.par", "a") as f:
        f.write("image1par = img1.par\n")
    r = _run(tools["strack"], ["track.par"], tmp_path)
    assert r.returncode == 1 and "VRT" in r.stderr


def test_parsing_reaches_the_device(tools, tmp_path, pair):
    """Without a GPU the tools stop exactly when the device is needed."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    a, b = pair
    _setup_track(tmp_path, a, b)
    r = _run(tools["strack"], ["-LSB", "track.par"], tmp_path)
    assert r.returncode == 1 and "CUDA device" in r.stderr


@pytest.mark.gpu
def test_strack_cli_matches_library(tools, tmp_path, pair):
    from specklesource_b200 import runtime
    a, b = pair
    kv = _setup_track(tmp_path, a, b)
    r = _run(tools["strack"], ["track.par"], tmp_path)
    assert r.returncode == 0, r.stderr
    out = files.read_track_outputs(str(tmp_path / "out"), kv["nR"], kv["nA"])
    p = abi.TrackParams(rStart=40, aStart=40, deltaR=16, deltaA=8, nR=27, nA=25, wR=32, wA=32, wRa=32, wAa=32)
    with runtime.Context(0, tuning=False) as ctx:  # the tools run the default launch shapes
        g = ctx.strack(p, a, b)
    for k, q in (("dr", "offR"), ("da", "offA"), ("cc", "corr"), ("azd", "azd"), ("mt", "type")):
        assert np.array_equal(out[k], g[q]), k
    dat = (tmp_path / "out.dat").read_text().split("\n")
    assert dat[0].split() == ["40", "40", "27", "25", "16", "8"]
    assert dat[1].split()[0] == "dummy.geodat"
    vrt = (tmp_path / "out.vrt").read_text()
    assert 'rasterXSize="27"' in vrt and "RangeOffsets" in vrt and "<ByteOrder>MSB</ByteOrder>" in vrt
    # little-endian images (VRT ByteOrder LSB, which like the reference sets the
    # byte order of the outputs too): same values in little-endian files
    files.write_slc(str(tmp_path / "img1.slc"), a, byte_order="LSB")
    files.write_slc(str(tmp_path / "img2.slc"), b, byte_order="LSB")
    r = _run(tools["strack"], ["-LSB", "track.par"], tmp_path)
    assert r.returncode == 0, r.stderr
    out2 = files.read_track_outputs(str(tmp_path / "out"), kv["nR"], kv["nA"], byte_order="LSB")
    assert np.array_equal(out2["dr"], g["offR"])


@pytest.mark.gpu
def test_strack_cli_flags_reach_the_library(tools, tmp_path, pair):
    """-gauss, -noComplex with -singleAmp, -noHanning and -checkAzFocus set the
    same parameters as the reference's flags (strack.c readArgs): the tool's
    files equal the library's results for those parameters."""
    from specklesource_b200 import runtime
    a, b = pair
    kv = _setup_track(tmp_path, a, b)
    base = dict(rStart=40, aStart=40, deltaR=16, deltaA=8, nR=27, nA=25, wR=32, wA=32, wRa=32, wAa=32)
    cases = [(["-gauss"], dict(gaussFlag=1)),
             (["-noComplex", "-singleAmp"], dict(noComplex=1, maxTries=1)),
             (["-noHanning", "-checkAzFocus"], dict(hanningFlag=0, checkAzFocus=1))]
    with runtime.Context(0, tuning=False) as ctx:  # the tools run the default launch shapes
        for flags, kw in cases:
            r = _run(tools["strack"], flags + ["track.par"], tmp_path)
            assert r.returncode == 0, r.stderr
            out = files.read_track_outputs(str(tmp_path / "out"), kv["nR"], kv["nA"])
            g = ctx.strack(abi.TrackParams(**base, **kw), a, b)
            for k, q in (("dr", "offR"), ("da", "offA"), ("cc", "corr"), ("mt", "type")):
                assert np.array_equal(out[k], g[q]), (flags, k)
            assert (g["type"] > 0).mean() > 0.9, flags


@pytest.mark.gpu
def test_strackw_and_cullst_cli(tools, tmp_path, pair):
    from specklesource_b200 import runtime
    a, b = pair
    _setup_track(tmp_path, a, b, wra=64, waa=64, edgepad=8, navgR=2, navgA=2, rstart=48, astart=48, deltar=24,
                 deltaa=24, nR=18, nA=7)
    r = _run(tools["strackw"], ["track.par"], tmp_path)
    assert r.returncode == 0, r.stderr
    out = files.read_track_outputs(str(tmp_path / "out"), 18, 7, azd=False)
    p = abi.TrackParams(rStart=48, aStart=48, deltaR=24, deltaA=24, nR=18, nA=7, wR=32, wA=32, wRa=64, wAa=64,
                        edgePadR=8, edgePadA=8, navgR=2, navgA=2)
    with runtime.Context(0, tuning=False) as ctx:  # the tools run the default launch shapes
        g = ctx.strackw(p, a, b)
        assert np.array_equal(out["dr"], g["offR"]) and np.array_equal(out["mt"], g["type"])
        # cullst on a synthetic offsets grid written in the reference's format
        rng = np.random.default_rng(2)
        nA, nR = 60, 80
        offR = (2 + 0.1 * rng.standard_normal((nA, nR))).astype(np.float32)
        offA = (0.5 + 0.1 * rng.standard_normal((nA, nR))).astype(np.float32)
        offR[rng.random((nA, nR)) < 0.08] += 15
        corr = rng.uniform(0.2, 0.9, (nA, nR)).astype(np.float32)
        mt = np.ones((nA, nR), np.uint8)
        files.write_offsets(str(tmp_path / "in"), offR, offA, corr, mt, 100, 200, 16, 8)
        r = _run(tools["cullst"], ["-islandThresh", "5", "-sr", "3", "-sa", "3", "in", "culled"], tmp_path)
        assert r.returncode == 0, r.stderr
        cp = abi.CullParams(nR=nR, nA=nA, islandThresh=5, sR=3, sA=3)
        d = ctx.cull(cp, offR, offA, corr, mt)
    assert np.array_equal(files.read_grid(str(tmp_path / "culled.dr"), nR, nA), d["offRS"])
    assert np.array_equal(files.read_grid(str(tmp_path / "culled.da"), nR, nA), d["offAS"])
    assert np.array_equal(files.read_grid(str(tmp_path / "in.sr"), nR, nA), d["sigmaR"])
    assert os.path.exists(tmp_path / "culled.vrt") and os.path.exists(tmp_path / "culled.mt.vrt")


@pytest.mark.gpu
def test_strack_cli_interferogram(tools, tmp_path):
    """intfile: the interferogram (big-endian CInt16 with looks in its VRT)
    flattens the fringe exactly as the library call does; a short file's
    missing lines hold (1, 1) like getInt's fill."""
    import torch
    from specklesource_b200 import runtime
    s1, s2 = synth.make_pair(256, 512, 11, dr=lambda y, x: 1.3 + 0 * x, da=lambda y, x: 0.4 + 0 * x,
                             coherence=0.8, ramp=0.6)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    kv = _setup_track(tmp_path, a, b, rstart=40, astart=40, deltar=16, deltaa=16, nR=27, nA=12)
    intf = synth.fringe_interferogram(256, 512, 4, 2, 0.6)
    files.write_interferogram(str(tmp_path / "int.int"), intf, 4, 2, lines=100)
    with open(tmp_path / "track.par", "a") as f:
        f.write("intfile = int.int\n")
    r = _run(tools["strack"], ["track.par"], tmp_path)
    assert r.returncode == 0, r.stderr
    out = files.read_track_outputs(str(tmp_path / "out"), kv["nR"], kv["nA"])
    full = intf.copy()
    full[100:] = np.array([1, 1], ">i2")
    p = abi.TrackParams(rStart=40, aStart=40, deltaR=16, deltaA=16, nR=27, nA=12, wR=32, wA=32, wRa=32, wAa=32,
                        intf=dict(data=full, nrl=4, nal=2))
    with runtime.Context(0, tuning=False) as ctx:  # the tools run the default launch shapes
        g = ctx.strack(p, a, b)
    for k, q in (("dr", "offR"), ("da", "offA"), ("mt", "type")):
        assert np.array_equal(out[k], g[q]), k
    assert (g["type"][:6] == 1).all()  # rows whose interferogram patches lie in the file's 100 lines


@pytest.mark.gpu
def test_initial_offsets_from_vrt_or_dat(tools, tmp_path, pair):
    """initShift: the offsets VRT (range and azimuth bands with r0/a0/deltaR/
    deltaA metadata, readBothOffsetsStrackVrt) and the .da/.dr/.dat files
    (readBothOffsetsStrack) give the same run."""
    a, b = pair
    _setup_track(tmp_path, a, b, outputfile="prev")
    r = _run(tools["strack"], ["track.par"], tmp_path)
    assert r.returncode == 0, r.stderr
    txt = (tmp_path / "track.par").read_text().replace("outputfile = prev", "outputfile = out")
    (tmp_path / "track.par").write_text(txt + "initShift = prev\n")
    r = _run(tools["strack"], ["track.par"], tmp_path)
    assert r.returncode == 0, r.stderr
    via_vrt = files.read_track_outputs(str(tmp_path / "out"), 27, 25)
    os.remove(tmp_path / "prev.vrt")
    # the older route reads <initShift>.da.dat, as readBothOffsetsStrack does
    (tmp_path / "prev.da.dat").write_text((tmp_path / "prev.dat").read_text())
    r = _run(tools["strack"], ["track.par"], tmp_path)
    assert r.returncode == 0, r.stderr
    via_dat = files.read_track_outputs(str(tmp_path / "out"), 27, 25)
    for k in ("dr", "da", "mt"):
        assert np.array_equal(via_vrt[k], via_dat[k]), k
    assert (via_vrt["mt"] > 0).mean() > 0.9
