"""TEST INFRASTRUCTURE ONLY: runs the reference's own tracking and culling
code, compiled unmodified from the reference tree against the stand-ins in
oracle/refshim/ (oracle/_ref/ref_strack, ref_strackw, ref_cull; built by
`make -C oracle ref` where the reference tree is present), so that the oracle
restatement can be checked against it.

Each call runs the binary in its own process (the reference keeps its state in
module globals and never frees it) on files in a temporary directory: raw
native-order images, a "key value" parameter file, and optional offset-grid
and mask files; the outputs are the reference's own .dr .da .cc .mt (.azd)
files.  Only tests/ and tests/golden/make_ref_golden.py use this.
"""
import os
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def available(tool="ref_strack"):
    return os.path.exists(os.path.join(REF_DIR, tool))


def _image_file(d, name, img):
    a = np.ascontiguousarray(img)
    if a.dtype == np.complex64 or a.dtype == np.dtype(">c8"):
        a = a.astype(np.complex64)
        float_flag = 1
    else:  # int16 (na, nr, 2): the reference always byte-swaps int16 samples
        a = a.astype(">i2")          # (loadBuffer, Strack/speckleTrack.c:1385-1388), so the file is big-endian
        float_flag = 0
    path = os.path.join(d, name)
    a.tofile(path)
    return path, a.shape[0], a.shape[1], float_flag


def _grids(out, nA, nR, azd=True):
    g = {k: np.fromfile(out + "." + k, dtype=np.float32).reshape(nA, nR) for k in ("dr", "da", "cc")}
    res = {"offR": g["dr"], "offA": g["da"], "corr": g["cc"],
           "type": np.fromfile(out + ".mt", dtype=np.uint8).reshape(nA, nR)}
    if azd:
        res["azd"] = np.fromfile(out + ".azd", dtype=np.float32).reshape(nA, nR)
    return res


_TRACK_KEYS = ("rStart", "aStart", "deltaR", "deltaA", "nR", "nA", "wR", "wA", "wRa", "wAa", "scaleFactor",
               "noComplex", "hanningFlag", "maxTries", "checkAzFocus", "gaussFlag", "azDefocusThresh", "polyShift",
               "edgePadR", "edgePadA", "navgR", "navgA")


def _track(tool, params, img1, img2, baseline=None, timeout=1800):
    """Runs ref_strack / ref_strackw on a TrackParams (specklesource_b200.abi)
    and two images; returns the output grids (and the baseline tables)."""
    with tempfile.TemporaryDirectory() as d:
        p1, na1, nr1, ff = _image_file(d, "img1", img1)
        p2, na2, nr2, _ = _image_file(d, "img2", img2)
        out = os.path.join(d, "out")
        lines = [f"image1 {p1}", f"image2 {p2}", f"out {out}", f"na1 {na1}", f"nr1 {nr1}", f"na2 {na2}",
                 f"nr2 {nr2}", f"floatFlag {ff}", "byteOrder 0"]
        for k in _TRACK_KEYS:
            lines.append(f"{k} {getattr(params, k)}")
        for i in range(3):
            lines.append(f"rpoly{i} {float(params.rShiftPoly[i])!r}")
            lines.append(f"apoly{i} {float(params.aShiftPoly[i])!r}")
        if params.initOffsets is not None:
            o = params.initOffsets
            of = os.path.join(d, "offsets")
            np.concatenate([np.ascontiguousarray(o["dr"], np.float32).ravel(),
                            np.ascontiguousarray(o["da"], np.float32).ravel()]).tofile(of)
            lines += [f"ofile {of}", f"onr {o['nr']}", f"ona {o['na']}", f"or0 {float(o['r0'])!r}",
                      f"oa0 {float(o['a0'])!r}", f"odeltaR {float(o['deltaR'])!r}",
                      f"odeltaA {float(o['deltaA'])!r}"]
        if params.mask is not None:
            m = params.mask
            mf = os.path.join(d, "mask")
            np.ascontiguousarray(m["mask"], np.uint8).tofile(mf)
            lines += [f"mfile {mf}", f"mnr {m['nr']}", f"mna {m['na']}", f"mr0 {m['r0']}", f"ma0 {m['a0']}",
                      f"mnrl {m['nrl']}", f"mnal {m['nal']}"]
        if baseline is not None:
            for k in ("Bn", "Bp", "dBn", "dBp", "dBnQ", "dBpQ", "lambda", "H", "rn", "slpR", "latc"):
                if k in baseline:
                    lines.append(f"{k} {float(baseline[k])!r}")
        pf = os.path.join(d, "params")
        with open(pf, "w") as f:
            f.write("\n".join(lines) + "\n")
        r = subprocess.run([os.path.join(REF_DIR, tool), pf], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"{tool} failed ({r.returncode}): {r.stderr[-2000:]}")
        res = _grids(out, params.nA, params.nR, azd=(tool == "ref_strack"))
        st = dict(zip(r.stdout.split()[0::2], map(int, r.stdout.split()[1::2])))
        res["stats"] = st
        tp = out + ".tables"
        if os.path.exists(tp):
            t = np.fromfile(tp, dtype=np.float64).reshape(3, nr1)
            res["tables"] = {"sinThetaD": t[0], "cosThetaD": t[1], "overRange": t[2]}
        return res


def strack(params, img1, img2, baseline=None):
    """The reference's speckleTrack() on two images (complex64 (na, nr) or
    int16 (na, nr, 2)).  baseline: Bn, Bp, dBn, dBp, dBnQ, dBpQ, lambda and
    the geometry H, rn, slpR, latc from which initPhaseCorrect tabulates the
    look angles (defaults give finite tables and a zero baseline)."""
    return _track("ref_strack", params, img1, img2, baseline)


def strackw(params, img1, img2):
    """The reference's corrTrackFast() on two images."""
    return _track("ref_strackw", params, img1, img2)


def cull(params, offR, offA, corr, mtype, mask=None, simR=None, simA=None, timeout=600):
    """The reference's cull passes in cullst's order (ref_cull) on a
    CullParams (specklesource_b200.abi); returns the culled, smoothed and
    sigma grids."""
    nA, nR = offR.shape
    with tempfile.TemporaryDirectory() as d:
        base = os.path.join(d, "in")
        out = os.path.join(d, "out")
        np.ascontiguousarray(offR, np.float32).tofile(base + ".offR")
        np.ascontiguousarray(offA, np.float32).tofile(base + ".offA")
        np.ascontiguousarray(corr, np.float32).tofile(base + ".corr")
        np.ascontiguousarray(mtype, np.uint8).tofile(base + ".type")
        if mask is not None:
            np.ascontiguousarray(mask, np.uint8).tofile(base + ".mask")
        if params.useSim:
            np.ascontiguousarray(simR, np.float32).tofile(base + ".simR")
            np.ascontiguousarray(simA, np.float32).tofile(base + ".simA")
        lines = [f"in {base}", f"out {out}", f"nR {nR}", f"nA {nA}", f"passes {params.nCullPasses}",
                 f"connectivity {params.connectivity}"]
        for k in ("bR", "bA", "nGood", "maxA", "maxR", "sR", "sA", "islandThresh", "corrThresh", "singleMT",
                  "useSim"):
            v = getattr(params, k)
            lines.append(f"{k} {float(v)!r}" if isinstance(v, float) else f"{k} {v}")
        pf = os.path.join(d, "params")
        with open(pf, "w") as f:
            f.write("\n".join(lines) + "\n")
        r = subprocess.run([os.path.join(REF_DIR, "ref_cull"), pf], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_cull failed ({r.returncode}): {r.stderr[-2000:]}")
        res = {k: np.fromfile(out + "." + k, dtype=np.float32).reshape(nA, nR)
               for k in ("offR", "offA", "offRS", "offAS", "sigmaR", "sigmaA")}
        res["type"] = np.fromfile(out + ".type", dtype=np.uint8).reshape(nA, nR)
        return res
