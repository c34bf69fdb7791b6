"""Writes tests/golden/ref_small.npz: outputs of the REFERENCE'S OWN CODE on
small seeded cases -- speckleTrack (Strack/speckleTrack.c), corrTrackFast
(Strackw/corrTrackFast.c) and the cull passes (Cullst/cull*.c), compiled
unmodified from the reference tree against oracle/refshim/ (`make -C oracle
ref`, run by oracle/refpin.py) -- so that tests/test_ref_pin.py can check the
oracle against the reference where the reference tree is absent.  The inputs
are regenerated from their seeds by the test.  Run from the repository root
where the reference tree is present:

    python tests/golden/make_ref_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def inputs():
    """The seeded inputs of every case (shared with the test)."""
    from specklesource_b200 import abi, synth
    s1, s2 = synth.small_pair(na=256, nr=384, seed=5)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    l1, l2 = synth.make_pair(256, 384, 21, dr=lambda y, x: 1.3 + 0 * x, da=lambda y, x: -0.6 + 0 * y,
                             coherence=0.25)
    la, lb = synth.to_numpy(l1), synth.to_numpy(l2)
    ai = np.stack([np.round(a.real * 3000), np.round(a.imag * 3000)], -1).astype(np.int16)
    bi = np.stack([np.round(b.real * 3000), np.round(b.imag * 3000)], -1).astype(np.int16)
    grid = dict(rStart=40, aStart=40, deltaR=24, deltaA=24, nR=11, nA=7, wR=32, wA=32, wRa=32, wAa=32)
    track = {
        "strack": (abi.TrackParams(**grid), a, b),
        "amp": (abi.TrackParams(**grid, noComplex=1), a, b),
        "lowcoh": (abi.TrackParams(**dict(grid, rStart=64, aStart=64, deltaR=16, deltaA=16, nR=16, nA=9)), la, lb),
        "gauss": (abi.TrackParams(**grid, gaussFlag=1), a, b),
        "int16": (abi.TrackParams(**grid), ai, bi),
    }
    pw = abi.TrackParams(rStart=80, aStart=80, deltaR=48, deltaA=48, nR=4, nA=2, wR=64, wA=64, wRa=64, wAa=64,
                         edgePadR=8, edgePadA=8, navgR=2, navgA=2)
    offR, offA, corr, mt = synth.offsets_field(40, 60, 3)
    cp = abi.CullParams(nR=60, nA=40, bR=5, bA=5, nGood=12, sR=3, sA=3, islandThresh=4)
    return track, (pw, a, b), (cp, offR, offA, corr, mt)


def cases():
    from oracle import oracle, refpin
    from specklesource_b200 import abi
    track, (pw, a, b), (cp, offR, offA, corr, mt) = inputs()
    out = {}
    for name, (p, x, y) in track.items():
        r = refpin.strack(p, x, y)
        for k in ("offR", "offA", "corr", "type", "azd"):
            out[f"{name}_{k}"] = r[k]
    r = refpin.strackw(pw, a, b)
    for k in ("offR", "offA", "corr", "type"):
        out[f"strackw_{k}"] = r[k]
    # the reference's stats, smoothing and island passes on the oracle's
    # culled grid (the median pass is compared separately: see the test)
    o = oracle.cull(cp, offR, offA, corr, mt, passes=("st", "st", "st"))
    cp0 = abi.CullParams(**{k: getattr(cp, k) for k in vars(cp)})
    cp0.nCullPasses = 0
    r = refpin.cull(cp0, o["offR"], o["offA"], corr, o["type"])
    for k in ("offRS", "offAS", "sigmaR", "sigmaA"):
        out[f"cull_{k}"] = r[k]
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_small.npz"), **cases())
    print("written")
