"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (oracle/lib/*.so).

Pinned to the reference's own code: tests/test_ref_pin.py compares it with the
reference's hot-path sources compiled against oracle/refshim/ (oracle/refpin.py)
and with committed outputs of that build; known-answer tests of its own are in
tests/test_oracle_kat.py.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from specklesource_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def build():
    """Compile both oracle libraries (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(precision="f64"):
    if precision not in _LIBS:
        path = os.path.join(_HERE, "lib", f"liboracle_{precision}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        for name in ("oracle_strack", "oracle_strackw"):
            f = getattr(L, name)
            f.argtypes = [C.POINTER(abi.SbTrackParams), C.POINTER(abi.SbImage), C.POINTER(abi.SbImage),
                          C.POINTER(abi.SbTrackResult), C.c_int32, C.c_int32]
            f.restype = C.c_int
        for name in ("oracle_cull", "oracle_cull_st_data", "oracle_cull_stats", "oracle_cull_smooth",
                     "oracle_cull_islands"):
            f = getattr(L, name)
            f.argtypes = [C.POINTER(abi.SbCullParams), C.POINTER(abi.SbCullData)]
            f.restype = C.c_int
        L.oracle_cullls.argtypes = [C.POINTER(abi.SbCulllsParams), C.POINTER(abi.SbCulllsData)]
        L.oracle_cullls.restype = C.c_int
        L.oracle_est_dop_carrier.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32]
        L.oracle_est_dop_carrier.restype = C.c_int
        L.oracle_fft2d.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]
        L.oracle_fft2d.restype = C.c_int
        L.oracle_fft2d_time.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
        L.oracle_fft2d_time.restype = C.c_int
        L.oracle_real_size.restype = C.c_int
        _LIBS[precision] = L
    return _LIBS[precision]


def _track(fn, params, img1, img2, rows=None, azd=True):
    p, keep = params.to_c()
    i1 = abi.make_image(img1)
    i2 = abi.make_image(img2)
    out, r = abi.alloc_track_result(params.nA, params.nR, azd=azd)
    r0, r1 = (0, 0) if rows is None else rows
    rc = fn(C.byref(p), C.byref(i1), C.byref(i2), C.byref(r), r0, r1)
    if rc != abi.SB_OK:
        raise RuntimeError(f"oracle returned {rc}")
    out["stats"] = abi.stats_of(r)
    return out


def strack(params, img1, img2, precision="f64", rows=None):
    """speckleTrack restated on the CPU. Images: complex64 (na, nr) arrays,
    native or big-endian ('>c8')."""
    return _track(lib(precision).oracle_strack, params, img1, img2, rows)


def strackw(params, img1, img2, precision="f64", rows=None):
    """corrTrackFast restated on the CPU."""
    return _track(lib(precision).oracle_strackw, params, img1, img2, rows, azd=False)


def _cull_data(offR, offA, corr, mtype, mask=None, simR=None, simA=None):
    nA, nR = offR.shape
    d = {
        "offR": np.array(offR, np.float32, copy=True),
        "offA": np.array(offA, np.float32, copy=True),
        "corr": np.ascontiguousarray(corr, np.float32),
        "type": np.array(mtype, np.uint8, copy=True),
        "mask": None if mask is None else np.ascontiguousarray(mask, np.uint8),
        "simR": None if simR is None else np.ascontiguousarray(simR, np.float32),
        "simA": None if simA is None else np.ascontiguousarray(simA, np.float32),
        "offRS": np.zeros((nA, nR), np.float32),
        "offAS": np.zeros((nA, nR), np.float32),
        "sigmaR": np.zeros((nA, nR), np.float32),
        "sigmaA": np.zeros((nA, nR), np.float32),
    }
    cd = abi.SbCullData(*[abi.ptr(d[k]) for k in ("offR", "offA", "corr", "type", "mask", "simR", "simA",
                                                  "offRS", "offAS", "sigmaR", "sigmaA")], 0, 0, 0, 0)
    return d, cd


def cull(params, offR, offA, corr, mtype, mask=None, simR=None, simA=None, passes=("all",)):
    """cullst pipeline (or selected passes: 'st', 'stats', 'smooth', 'islands')."""
    L = lib("f64")
    d, cd = _cull_data(offR, offA, corr, mtype, mask, simR, simA)
    p = params.to_c()
    fns = {"all": L.oracle_cull, "st": L.oracle_cull_st_data, "stats": L.oracle_cull_stats,
           "smooth": L.oracle_cull_smooth, "islands": L.oracle_cull_islands}
    for name in passes:
        rc = fns[name](C.byref(p), C.byref(cd))
        if rc != abi.SB_OK:
            raise RuntimeError(f"oracle cull returned {rc}")
    d["nCulled"] = cd.nCulled
    d["nIslands"] = cd.nIslands
    d["nIslandPoints"] = cd.nIslandPoints
    return d


def cullls(params, X, Y, mtype):
    """cullls pipeline (Cullls/cullls.c:23-56)."""
    d, cd = abi.cullls_data(X, Y, mtype)
    p = params.to_c()
    rc = lib("f64").oracle_cullls(C.byref(p), C.byref(cd))
    if rc != abi.SB_OK:
        raise RuntimeError(f"oracle cullls returned {rc}")
    for k in ("nAttempt", "nMatch", "nCulled", "nIslands", "nIslandPoints"):
        d[k] = getattr(cd, k)
    return d


def est_dop_carrier(p1, p2, wA):
    a = np.ascontiguousarray(p1, np.complex64)
    b = np.ascontiguousarray(p2, np.complex64)
    nAz, nRg = a.shape
    return lib("f64").oracle_est_dop_carrier(a.ctypes.data, b.ctypes.data, nAz, nRg, wA)


def fft2d_time(na, nr, reps, precision="f32"):
    """Seconds per forward na x nr transform of the restatement's FFT (plan
    made once, one thread)."""
    t = C.c_double(0.0)
    lib(precision).oracle_fft2d_time(na, nr, reps, C.byref(t))
    return t.value


def fft2d(x, sign=-1, precision="f64"):
    """Unnormalised 2-D DFT with the FFTW sign convention (sign -1 forward)."""
    a = np.ascontiguousarray(x, np.complex128).copy()
    na, nr = a.shape
    lib(precision).oracle_fft2d(a.ctypes.data, na, nr, sign)
    return a
