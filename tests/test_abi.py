"""C-ABI checks that need no GPU: the library loads, exports every function
declared in include/*.h, and the ctypes mirror matches the C struct layouts."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from specklesource_b200 import abi, build, runtime

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return runtime.load()


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(sb_[a-z0-9_]+)\s*\(", txt))
    return names


def test_every_declared_symbol_is_exported(lib):
    names = _declared_functions()
    assert len(names) >= 14
    out = subprocess.run(["nm", "-D", "--defined-only", runtime.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (sb_[a-z0-9_]+)", out))
    missing = names - exported
    assert not missing, f"declared but not exported: {missing}"
    assert names <= set(runtime.SIGNATURES), "runtime.SIGNATURES lacks a declared function"
    for n in names:
        assert hasattr(lib, n)


def test_abi_version(lib):
    assert lib.sb_abi_version() == 2


def test_context_without_device_reports_error(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    rc = lib.sb_context_create(0, C.byref(h))
    assert rc == abi.SB_ERR_NODEVICE and not h.value


_STRUCTS = {
    "sb_image": abi.SbImage,
    "sb_offset_grid": abi.SbOffsetGrid,
    "sb_mask": abi.SbMask,
    "sb_baseline": abi.SbBaseline,
    "sb_interferogram": abi.SbInterferogram,
    "sb_track_params": abi.SbTrackParams,
    "sb_track_result": abi.SbTrackResult,
    "sb_cull_params": abi.SbCullParams,
    "sb_cull_data": abi.SbCullData,
    "sb_cullls_params": abi.SbCulllsParams,
    "sb_cullls_data": abi.SbCulllsData,
}


def test_ctypes_layout_matches_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "speckle_b200.h"', "int main(void){"]
    for cname, cls in _STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            cf = "lambda" if fname == "lambda_" else fname
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {cf}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            s, f, v = ln.split()
            got[(s, f)] = int(v)
    for cname, cls in _STRUCTS.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_peak_hand_off_constants_agree(tmp_path):
    """The complex stage's list chunk and PeakJob size, as the library defines
    them, are the figures bench.py and the job server's memory estimate use."""
    import re

    import bench
    from specklesource_b200 import serve
    src = open(os.path.join(ROOT, "specklesource_b200", "csrc", "capi.cu")).read()
    chunk = 1 << int(re.search(r"kPeakChunk = 1 << (\d+);", src).group(1))
    assert chunk == bench.PEAK_CHUNK == serve._PEAK_CHUNK
    prog = tmp_path / "pj.cu"
    prog.write_text('#include <cstdio>\n#include "strack_kernels.h"\n'
                    'int main() { std::printf("%zu\\n", sizeof(sbk::PeakJob)); return 0; }\n')
    exe = tmp_path / "pj"
    subprocess.run(["nvcc", "-std=c++17", "-I", os.path.join(ROOT, "specklesource_b200", "csrc"), str(prog), "-o",
                    str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert int(out) == serve._PEAK_JOB_BYTES
