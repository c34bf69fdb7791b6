"""ctypes mirror of include/speckle_b200.h (the library's C ABI).

Only plain C types appear here; the structs match the header field for field.
"""
import ctypes as C

import numpy as np

SB_OK = 0
SB_ERR_ARG = -1
SB_ERR_CUDA = -2
SB_ERR_NOMEM = -3
SB_ERR_UNSUPPORTED = -4
SB_ERR_NODEVICE = -5
SB_ERR_TIMEOUT = -6
SB_FORM_FP32 = 0
SB_FORM_SPLIT_BF16 = 1
SB_TUNE_COMPLEX = 0
SB_TUNE_COMPLEX_TC = 1
SB_TUNE_AMPLITUDE = 2

SB_LARGEINT = 2000000000
SB_BAD, SB_CMATCH, SB_AMPMATCH, SB_AMPMATCHLARGE = 0, 1, 2, 3
SB_LSB, SB_MSB = 0, 1
SB_CFLOAT32, SB_CINT16 = 0, 1

_i32 = C.c_int32
_i64 = C.c_int64
_f32 = C.c_float
_f64 = C.c_double


class SbImage(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("nr", _i32),
        ("na", _i32),
        ("sampleType", _i32),
        ("byteOrder", _i32),
        ("onDevice", _i32),
    ]


class SbOffsetGrid(C.Structure):
    _fields_ = [
        ("nr", _i32),
        ("na", _i32),
        ("r0", _f64),
        ("a0", _f64),
        ("deltaR", _f64),
        ("deltaA", _f64),
        ("dr", C.c_void_p),
        ("da", C.c_void_p),
    ]


class SbMask(C.Structure):
    _fields_ = [
        ("r0", _i32),
        ("a0", _i32),
        ("nr", _i32),
        ("na", _i32),
        ("nrl", _i32),
        ("nal", _i32),
        ("mask", C.c_void_p),
    ]


class SbBaseline(C.Structure):
    _fields_ = [
        ("Bn", _f64), ("Bp", _f64), ("dBn", _f64), ("dBp", _f64), ("dBnQ", _f64), ("dBpQ", _f64),
        ("lambda_", _f64),
        ("sinThetaD", C.c_void_p),
        ("cosThetaD", C.c_void_p),
        ("overRange", C.c_void_p),
    ]


class SbInterferogram(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("nr", _i32), ("na", _i32),
        ("nrl", _i32), ("nal", _i32),
        ("byteOrder", _i32),
        ("onDevice", _i32),
    ]


class SbTrackParams(C.Structure):
    _fields_ = [
        ("rStart", _i32), ("aStart", _i32),
        ("deltaR", _i32), ("deltaA", _i32),
        ("nR", _i32), ("nA", _i32),
        ("wR", _i32), ("wA", _i32),
        ("wRa", _i32), ("wAa", _i32),
        ("scaleFactor", _i32),
        ("noComplex", _i32),
        ("hanningFlag", _i32),
        ("maxTries", _i32),
        ("checkAzFocus", _i32),
        ("gaussFlag", _i32),
        ("azDefocusThresh", _f32),
        ("edgePadR", _i32), ("edgePadA", _i32),
        ("navgR", _i32), ("navgA", _i32),
        ("polyShift", _i32),
        ("rShiftPoly", _f64 * 3),
        ("aShiftPoly", _f64 * 3),
        ("initOffsets", C.POINTER(SbOffsetGrid)),
        ("mask", C.POINTER(SbMask)),
        ("baseline", C.POINTER(SbBaseline)),
        ("intf", C.POINTER(SbInterferogram)),
    ]


class SbTrackResult(C.Structure):
    _fields_ = [
        ("offR", C.c_void_p),
        ("offA", C.c_void_p),
        ("corr", C.c_void_p),
        ("azd", C.c_void_p),
        ("type", C.c_void_p),
        ("onDevice", _i32),
        ("nComplex", _i64),
        ("nAmp", _i64),
        ("nAmpL", _i64),
        ("nFail", _i64),
        ("nAttempted", _i64),
    ]


class SbCullParams(C.Structure):
    _fields_ = [
        ("nR", _i32), ("nA", _i32),
        ("bR", _i32), ("bA", _i32),
        ("nGood", _i32),
        ("maxA", _f32), ("maxR", _f32),
        ("sR", _i32), ("sA", _i32),
        ("islandThresh", _i32),
        ("corrThresh", _f32),
        ("singleMT", _i32),
        ("useSim", _i32),
        ("connectivity", _i32),
        ("nCullPasses", _i32),
    ]


class SbCullData(C.Structure):
    _fields_ = [
        ("offR", C.c_void_p), ("offA", C.c_void_p),
        ("corr", C.c_void_p),
        ("type", C.c_void_p),
        ("mask", C.c_void_p),
        ("simR", C.c_void_p), ("simA", C.c_void_p),
        ("offRS", C.c_void_p), ("offAS", C.c_void_p),
        ("sigmaR", C.c_void_p), ("sigmaA", C.c_void_p),
        ("onDevice", _i32),
        ("nCulled", _i64),
        ("nIslands", _i64),
        ("nIslandPoints", _i64),
    ]


class SbCulllsParams(C.Structure):
    _fields_ = [
        ("nx", _i32), ("ny", _i32),
        ("boxSize", _i32),
        ("nGood", _i32),
        ("maxX", _f32), ("maxY", _f32),
        ("sX", _i32), ("sY", _i32),
        ("islandThresh", _i32),
        ("nCullPasses", _i32),
        ("connectivity", _i32),
        ("deltaT", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double),
        ("noDataLimit", C.c_double),
        ("nOver", C.c_double),
        ("slowVelMask", C.c_uint8),
        ("noDataMask", C.c_uint8),
        ("reserved", C.c_uint8 * 6),
    ]


class SbCulllsData(C.Structure):
    _fields_ = [
        ("X", C.c_void_p), ("Y", C.c_void_p),
        ("type", C.c_void_p),
        ("XS", C.c_void_p), ("YS", C.c_void_p),
        ("sigmaX", C.c_void_p), ("sigmaY", C.c_void_p),
        ("onDevice", _i32),
        ("nAttempt", _i64),
        ("nMatch", _i64),
        ("nCulled", _i64),
        ("nIslands", _i64),
        ("nIslandPoints", _i64),
    ]


def ptr(a):
    """Address of a numpy array (or None)."""
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return a.ctypes.data


# ---------------------------------------------------------------------------
# Python-level parameter objects (names as in TrackParams / CullParams)
# ---------------------------------------------------------------------------


class TrackParams:
    """Mirror of the reference's TrackParams for strack/strackw (Strack/strack.h:56-165).

    Defaults are those of the reference CLIs (Strack/strack.c:137-178,
    Strack/parseTrack.c:222-253).
    """

    def __init__(self, **kw):
        self.rStart = 0
        self.aStart = 0
        self.deltaR = 1
        self.deltaA = 1
        self.nR = 1
        self.nA = 1
        self.wR = 32
        self.wA = 32
        self.wRa = 32
        self.wAa = 32
        self.scaleFactor = 1
        self.noComplex = 0
        self.hanningFlag = 1
        self.maxTries = 2
        self.checkAzFocus = 0
        self.gaussFlag = 0
        self.azDefocusThresh = 1.8
        self.edgePadR = 0
        self.edgePadA = 0
        self.navgR = 1
        self.navgA = 1
        self.polyShift = 1
        self.rShiftPoly = (0.0, 0.0, 0.0)
        self.aShiftPoly = (0.0, 0.0, 0.0)
        self.initOffsets = None  # dict(nr, na, r0, a0, deltaR, deltaA, dr, da)
        self.mask = None  # dict(r0, a0, nr, na, nrl, nal, mask)
        self.intf = None  # dict(data=int16 (na, nr, 2) array, nrl, nal[, byteOrder])
        # dict(Bn, Bp, dBn, dBp, dBnQ, dBpQ, lambda_, sinThetaD, cosThetaD, overRange): the
        # baseparams terms and initPhaseCorrect's per-range-sample tables (speckleTrack.c:1556-1625)
        self.baseline = None
        for k, v in kw.items():
            if not hasattr(self, k):
                raise TypeError(f"unknown track parameter {k!r}")
            setattr(self, k, v)

    def to_c(self):
        """Returns (SbTrackParams, keepalive list)."""
        p = SbTrackParams()
        keep = []
        for name, _ in SbTrackParams._fields_:
            if name in ("rShiftPoly", "aShiftPoly", "initOffsets", "mask", "baseline", "intf"):
                continue
            setattr(p, name, getattr(self, name))
        for i in range(3):
            p.rShiftPoly[i] = float(self.rShiftPoly[i])
            p.aShiftPoly[i] = float(self.aShiftPoly[i])
        if self.initOffsets is not None:
            o = self.initOffsets
            dr = np.ascontiguousarray(o["dr"], dtype=np.float32)
            da = np.ascontiguousarray(o["da"], dtype=np.float32)
            g = SbOffsetGrid(int(o["nr"]), int(o["na"]), float(o["r0"]), float(o["a0"]),
                             float(o["deltaR"]), float(o["deltaA"]), ptr(dr), ptr(da))
            keep += [dr, da, g]
            p.initOffsets = C.pointer(g)
        if self.mask is not None:
            m = self.mask
            mk = np.ascontiguousarray(m["mask"], dtype=np.uint8)
            sm = SbMask(int(m["r0"]), int(m["a0"]), int(m["nr"]), int(m["na"]), int(m["nrl"]),
                        int(m["nal"]), ptr(mk))
            keep += [mk, sm]
            p.mask = C.pointer(sm)
        if self.baseline is not None:
            bl = self.baseline
            tabs = [np.ascontiguousarray(bl[k], dtype=np.float64) for k in ("sinThetaD", "cosThetaD", "overRange")]
            sb = SbBaseline(*[float(bl[k]) for k in ("Bn", "Bp", "dBn", "dBp", "dBnQ", "dBpQ", "lambda_")],
                            *[ptr(t) for t in tabs])
            keep += tabs + [sb]
            p.baseline = C.pointer(sb)
        if self.intf is not None:
            f = self.intf
            d = f["data"]
            if isinstance(d, np.ndarray):
                d = np.ascontiguousarray(d)
                order = SB_MSB if d.dtype.byteorder == ">" else SB_LSB
                na, nr = d.shape[:2]
                g = SbInterferogram(ptr(d), nr, na, int(f["nrl"]), int(f["nal"]), f.get("byteOrder", order), 0)
            else:  # torch CUDA int16 tensor (na, nr, 2), native order
                na, nr = d.shape[:2]
                g = SbInterferogram(d.data_ptr(), nr, na, int(f["nrl"]), int(f["nal"]), f.get("byteOrder", SB_LSB),
                                    1)
            keep += [d, g]
            p.intf = C.pointer(g)
        return p, keep


class CullParams:
    """Mirror of the reference's CullParams (Cullst/cullst.h:4-59) with the
    cullst CLI defaults (Cullst/cullst.c:133-145)."""

    def __init__(self, **kw):
        self.nR = 0
        self.nA = 0
        self.bR = 9
        self.bA = 9
        self.nGood = 17
        self.maxA = 1.0
        self.maxR = 0.75
        self.sR = 2
        self.sA = 8
        self.islandThresh = -1
        self.corrThresh = 0.0
        self.singleMT = -1
        self.useSim = 0
        self.connectivity = 8
        self.nCullPasses = 3
        for k, v in kw.items():
            if not hasattr(self, k):
                raise TypeError(f"unknown cull parameter {k!r}")
            setattr(self, k, v)

    def to_c(self):
        p = SbCullParams()
        for name, _ in SbCullParams._fields_:
            setattr(p, name, getattr(self, name))
        return p


def cullls_data(X, Y, mtype):
    """Host buffers of one cullls job: copies of X, Y, type and zeroed
    outputs; returns (dict of arrays, SbCulllsData over them)."""
    ny, nx = X.shape
    d = {
        "X": np.array(X, np.float32, copy=True),
        "Y": np.array(Y, np.float32, copy=True),
        "type": np.array(mtype, np.uint8, copy=True),
        "XS": np.zeros((ny, nx), np.float32),
        "YS": np.zeros((ny, nx), np.float32),
        "sigmaX": np.zeros((ny, nx), np.float32),
        "sigmaY": np.zeros((ny, nx), np.float32),
    }
    cd = SbCulllsData(*[ptr(d[k]) for k in ("X", "Y", "type", "XS", "YS", "sigmaX", "sigmaY")], 0, 0, 0, 0, 0, 0)
    return d, cd


class CullLSParams:
    """Mirror of the reference's CullLSParams (Cullls/cullls.h:2-35) with the
    cullls CLI defaults (Cullls/cullls.c:184-191), plus the landsatSource64
    values cullls reads from headers that are not in the reference tree:
    deltaT (days), dx/dy (pixel size, m), slowVelMask (SLOWVEL), noDataMask
    (NODATATOUSE), noDataLimit (NODATA + 1) and nOver (lstrack's NOVER, no
    default: it must be given)."""

    def __init__(self, **kw):
        self.nx = 0
        self.ny = 0
        self.boxSize = 9
        self.nGood = 17
        self.maxX = 0.75
        self.maxY = 1.0
        self.sX = 3
        self.sY = 3
        self.islandThresh = -1
        self.nCullPasses = 3
        self.connectivity = 8
        self.deltaT = 0.0
        self.dx = 0.0
        self.dy = 0.0
        self.noDataLimit = -1999999999.0
        self.nOver = 0.0
        self.slowVelMask = 0
        self.noDataMask = 0
        for k, v in kw.items():
            if not hasattr(self, k):
                raise TypeError(f"unknown cullls parameter {k!r}")
            setattr(self, k, v)

    def to_c(self):
        p = SbCulllsParams()
        for name, _ in SbCulllsParams._fields_:
            if name != "reserved":
                setattr(p, name, getattr(self, name))
        return p


def make_image(arr, byte_order=SB_LSB):
    """SbImage for a host numpy array: complex64 (na, nr), or int16 (na, nr, 2),
    or raw big-endian bytes given as uint8 with an explicit shape tuple."""
    if arr.dtype == np.complex64:
        st = SB_CFLOAT32
        na, nr = arr.shape
    elif arr.dtype == np.int16:
        st = SB_CINT16
        na, nr = arr.shape[:2]
    elif arr.dtype == np.dtype(">c8"):
        st = SB_CFLOAT32
        na, nr = arr.shape
        byte_order = SB_MSB
    elif arr.dtype == np.dtype(">i2"):
        st = SB_CINT16
        na, nr = arr.shape[:2]
        byte_order = SB_MSB
    else:
        raise TypeError(f"unsupported image dtype {arr.dtype}")
    assert arr.flags["C_CONTIGUOUS"]
    return SbImage(arr.ctypes.data, nr, na, st, byte_order, 0)


def alloc_track_result(nA, nR, azd=True):
    """Host output grids + an SbTrackResult pointing at them."""
    out = {
        "offR": np.zeros((nA, nR), np.float32),
        "offA": np.zeros((nA, nR), np.float32),
        "corr": np.zeros((nA, nR), np.float32),
        "azd": np.zeros((nA, nR), np.float32) if azd else None,
        "type": np.zeros((nA, nR), np.uint8),
    }
    r = SbTrackResult(ptr(out["offR"]), ptr(out["offA"]), ptr(out["corr"]), ptr(out["azd"]),
                      ptr(out["type"]), 0, 0, 0, 0, 0, 0)
    return out, r


def stats_of(r):
    return {"nComplex": r.nComplex, "nAmp": r.nAmp, "nAmpL": r.nAmpL, "nFail": r.nFail,
            "nAttempted": r.nAttempted}
