"""Python binding of libspeckle_b200.so (the C ABI in include/speckle_b200.h).

There is no CPU fallback: if the library or a CUDA device is missing, the
calls raise.  Host numpy arrays are copied to the device inside the call;
torch CUDA tensors may be passed for images and outputs to stay on the device.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libspeckle_b200.so")

# every function declared in include/speckle_b200.h: name -> (restype, argtypes)
_P = C.c_void_p
SIGNATURES = {
    "sb_abi_version": (C.c_int, []),
    "sb_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "sb_context_destroy": (None, [_P]),
    "sb_last_error": (C.c_char_p, [_P]),
    "sb_last_timing": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "sb_last_launch_count": (C.c_int64, [_P]),
    "sb_last_stage_timing": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "sb_set_wait_limit": (C.c_int, [_P, C.c_int64]),
    "sb_set_form": (C.c_int, [_P, C.c_int]),
    "sb_context_device_bytes": (C.c_int64, [_P]),
    "sb_set_tuning": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    "sb_context_release": (C.c_int, [_P]),
    "sb_last_form": (C.c_int, [_P]),
    "sb_strack": (C.c_int, [_P, C.POINTER(abi.SbTrackParams), C.POINTER(abi.SbImage), C.POINTER(abi.SbImage),
                            C.POINTER(abi.SbTrackResult)]),
    "sb_strackw": (C.c_int, [_P, C.POINTER(abi.SbTrackParams), C.POINTER(abi.SbImage), C.POINTER(abi.SbImage),
                             C.POINTER(abi.SbTrackResult)]),
    "sb_strack_batch": (C.c_int, [_P, C.c_int32, C.POINTER(abi.SbTrackParams), C.POINTER(abi.SbImage),
                                  C.POINTER(abi.SbImage), C.POINTER(abi.SbTrackResult)]),
    "sb_est_dop_carrier": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P]),
    "sb_cull": (C.c_int, [_P, C.POINTER(abi.SbCullParams), C.POINTER(abi.SbCullData)]),
    "sb_cull_st_data": (C.c_int, [_P, C.POINTER(abi.SbCullParams), C.POINTER(abi.SbCullData)]),
    "sb_cull_stats": (C.c_int, [_P, C.POINTER(abi.SbCullParams), C.POINTER(abi.SbCullData)]),
    "sb_cull_smooth": (C.c_int, [_P, C.POINTER(abi.SbCullParams), C.POINTER(abi.SbCullData)]),
    "sb_cull_islands": (C.c_int, [_P, C.POINTER(abi.SbCullParams), C.POINTER(abi.SbCullData)]),
    "sb_cullls": (C.c_int, [_P, C.POINTER(abi.SbCulllsParams), C.POINTER(abi.SbCulllsData)]),
    "sb_amp_match_noalloc": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, _P, _P, _P, _P, _P]),
}

_lib = None


def load(path=LIB_PATH):
    """Loads the library (raises OSError if it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} not built: run `python -m specklesource_b200.build`")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class SpeckleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"speckle_b200 error {code}: {msg}")
        self.code = code


def _is_torch_cuda(x):
    try:
        import torch
        return isinstance(x, torch.Tensor) and x.is_cuda
    except ImportError:
        return False


def image_desc(img, byte_order=None):
    """SbImage for numpy (host) or torch CUDA (device) images.

    numpy: complex64 (na, nr) native, '>c8' big-endian, or int16 (na, nr, 2).
    torch: complex64 (na, nr) or uint8 raw bytes (na, nr*8) with byte_order.
    """
    if _is_torch_cuda(img):
        import torch
        assert img.is_contiguous()
        if img.dtype == torch.complex64:
            na, nr = img.shape
            return abi.SbImage(img.data_ptr(), nr, na, abi.SB_CFLOAT32, abi.SB_LSB if byte_order is None else byte_order, 1)
        if img.dtype == torch.uint8:
            na, nb = img.shape
            return abi.SbImage(img.data_ptr(), nb // 8, na, abi.SB_CFLOAT32,
                               abi.SB_MSB if byte_order is None else byte_order, 1)
        if img.dtype == torch.int16:
            na, nr, _ = img.shape
            return abi.SbImage(img.data_ptr(), nr, na, abi.SB_CINT16, abi.SB_LSB if byte_order is None else byte_order, 1)
        raise TypeError(f"unsupported tensor dtype {img.dtype}")
    d = abi.make_image(img)
    if byte_order is not None:
        d.byteOrder = byte_order
    return d


def _device_name(device):
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return None


class Context:
    """One CUDA device, one stream; mirrors the reference's TrackParams/CullParams entry points."""

    def __init__(self, device=0, tuning=None):
        """tuning: None applies the autotuner's table (specklesource_b200/
        tuning.json) when it was measured on a device of this name; False
        applies none; a dict applies that table."""
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.sb_context_create(int(device), C.byref(h))
        if rc != abi.SB_OK:
            raise SpeckleError(rc, "sb_context_create failed (no CUDA device?)")
        self.h = h
        self.tuning_applied = 0
        if tuning is not False:
            from . import autotune
            table = tuning if isinstance(tuning, dict) else autotune.load()
            if table and (isinstance(tuning, dict) or table.get("device") == _device_name(device)):
                self.tuning_applied = autotune.apply(self, table)

    def close(self):
        if getattr(self, "h", None):
            self.lib.sb_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != abi.SB_OK:
            msg = self.lib.sb_last_error(self.h)
            raise SpeckleError(rc, msg.decode() if msg else "")

    def timing(self):
        ms = (C.c_float * 4)()
        self.lib.sb_last_timing(self.h, ms)
        return {"total": ms[0], "h2d": ms[1], "kernels": ms[2], "d2h": ms[3]}

    def stage_timing(self):
        ms = (C.c_float * 8)()
        self.lib.sb_last_stage_timing(self.h, ms)
        return {"cmplx_ms": ms[0], "amp_small_ms": ms[1], "amp_large_ms": ms[2], "fit_ms": ms[3],
                "book_ms": ms[4], "n_cmplx": int(ms[5]), "n_amp_small": int(ms[6]), "n_amp_large": int(ms[7])}

    def launch_count(self):
        return int(self.lib.sb_last_launch_count(self.h))

    def device_bytes(self):
        """Device memory this context holds (grown buffers + tables), bytes."""
        return int(self.lib.sb_context_device_bytes(self.h))

    def release(self):
        """Frees the context's grown buffers (they grow again on the next call)."""
        self._check(self.lib.sb_context_release(self.h))

    def set_form(self, form):
        """Transform form of strack's complex stage: abi.SB_FORM_FP32 (default)
        or abi.SB_FORM_SPLIT_BF16 (tensor cores, complex window 64)."""
        self._check(self.lib.sb_set_form(self.h, int(form)))

    def last_form(self):
        return int(self.lib.sb_last_form(self.h))

    def _track(self, fn, params, img1, img2, out, azd):
        p, keep = params.to_c()
        i1 = image_desc(img1)
        i2 = image_desc(img2)
        if out is None:
            out, r = abi.alloc_track_result(params.nA, params.nR, azd=azd)
        else:
            r = _result_from(out)
        self._check(fn(self.h, C.byref(p), C.byref(i1), C.byref(i2), C.byref(r)))
        out["stats"] = abi.stats_of(r)
        return out

    def strack(self, params, img1, img2, out=None):
        """speckleTrack (Strack/speckleTrack.c:159) on the GPU."""
        return self._track(self.lib.sb_strack, params, img1, img2, out, True)

    def strack_batch(self, params, imgs1, imgs2):
        """speckleTrack on many pairs in one call (sb_strack_batch): lists of
        TrackParams and images; returns one result dict per pair."""
        n = len(params)
        if not (len(imgs1) == len(imgs2) == n) or n == 0:
            raise ValueError("params, imgs1 and imgs2 must be non-empty lists of the same length")
        keep, outs = [], []
        P = (abi.SbTrackParams * n)()
        I1 = (abi.SbImage * n)()
        I2 = (abi.SbImage * n)()
        R = (abi.SbTrackResult * n)()
        for k in range(n):
            pc, kp = params[k].to_c()
            keep.append(kp)
            P[k] = pc
            I1[k] = image_desc(imgs1[k])
            I2[k] = image_desc(imgs2[k])
            o, r = abi.alloc_track_result(params[k].nA, params[k].nR, azd=True)
            outs.append(o)
            R[k] = r
        self._check(self.lib.sb_strack_batch(self.h, n, P, I1, I2, R))
        for k in range(n):
            outs[k]["stats"] = abi.stats_of(R[k])
        return outs

    def strackw(self, params, img1, img2, out=None):
        """corrTrackFast (Strackw/corrTrackFast.c:89) on the GPU."""
        return self._track(self.lib.sb_strackw, params, img1, img2, out, False)

    def cull(self, params, offR, offA, corr, mtype, mask=None, simR=None, simA=None, passes=("all",)):
        """cullst pipeline (Cullst/cullst.c:71-101), or single passes."""
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
        cp = params.to_c()
        fns = {"all": self.lib.sb_cull, "st": self.lib.sb_cull_st_data, "stats": self.lib.sb_cull_stats,
               "smooth": self.lib.sb_cull_smooth, "islands": self.lib.sb_cull_islands}
        for name in passes:
            self._check(fns[name](self.h, C.byref(cp), C.byref(cd)))
        d["nCulled"] = cd.nCulled
        d["nIslands"] = cd.nIslands
        d["nIslandPoints"] = cd.nIslandPoints
        return d

    def cullls(self, params, X, Y, mtype):
        """cullls pipeline (Cullls/cullls.c:23-56) on the GPU."""
        d, cd = abi.cullls_data(X, Y, mtype)
        cp = params.to_c()
        self._check(self.lib.sb_cullls(self.h, C.byref(cp), C.byref(cd)))
        for k in ("nAttempt", "nMatch", "nCulled", "nIslands", "nIslandPoints"):
            d[k] = getattr(cd, k)
        return d


def _result_from(out):
    """SbTrackResult over caller-provided grids (numpy host or torch CUDA)."""
    dev = _is_torch_cuda(out["offR"])

    def addr(x):
        if x is None:
            return None
        return x.data_ptr() if dev else abi.ptr(x)

    return abi.SbTrackResult(addr(out["offR"]), addr(out["offA"]), addr(out["corr"]), addr(out.get("azd")),
                             addr(out["type"]), 1 if dev else 0, 0, 0, 0, 0, 0)
