"""Writes tests/golden/oracle_small.npz: the FP64 oracle's outputs on small
seeded cases (strack complex and amplitude-only, strackw, cullst), so that any
change to the oracle that moves its results is caught by
tests/test_golden.py.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def cases():
    from oracle import oracle
    from specklesource_b200 import abi, synth
    s1, s2 = synth.small_pair(na=256, nr=384, seed=5)
    a, b = synth.to_numpy(s1), synth.to_numpy(s2)
    out = {}
    p = abi.TrackParams(rStart=40, aStart=40, deltaR=24, deltaA=24, nR=11, nA=7, wR=32, wA=32, wRa=32, wAa=32)
    o = oracle.strack(p, a, b)
    for k in ("offR", "offA", "corr", "type"):
        out[f"strack_{k}"] = o[k]
    o = oracle.strack(abi.TrackParams(rStart=40, aStart=40, deltaR=24, deltaA=24, nR=11, nA=7, wR=32, wA=32,
                                      wRa=32, wAa=32, noComplex=1), a, b)
    for k in ("offR", "offA", "corr", "type"):
        out[f"amp_{k}"] = o[k]
    pw = abi.TrackParams(rStart=80, aStart=80, deltaR=48, deltaA=48, nR=4, nA=2, wR=64, wA=64, wRa=64, wAa=64,
                         edgePadR=8, edgePadA=8, navgR=2, navgA=2)
    o = oracle.strackw(pw, a, b)
    for k in ("offR", "offA", "corr", "type"):
        out[f"strackw_{k}"] = o[k]
    offR, offA, corr, mt = synth.offsets_field(40, 60, 3)
    c = oracle.cull(abi.CullParams(nR=60, nA=40, bR=5, bA=5, nGood=12, sR=3, sA=3, islandThresh=4), offR, offA,
                    corr, mt)
    for k in ("offR", "offA", "offRS", "offAS", "sigmaR", "sigmaA"):
        out[f"cull_{k}"] = c[k]
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_small.npz"), **cases())
    print("written")
