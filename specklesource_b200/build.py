"""Builds the CUDA library libspeckle_b200.so for sm_100a, in-tree.

    python -m specklesource_b200.build

Each csrc/*.cu is compiled to an object under specklesource_b200/_build/ and
linked into specklesource_b200/lib/libspeckle_b200.so (CUDA runtime linked
statically, so the library carries no runtime dependency beyond the driver).
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libspeckle_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2", f"-I{INCLUDE}",
                "-diag-suppress", "550,177"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                  glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj
    cmd = [NVCC] + FLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


HOST = os.path.join(HERE, "host")
BINDIR = os.path.join(HERE, "bin")
CC = os.environ.get("CC", "gcc")


def build_cli():
    """The drop-in command lines strack, strackw and cullst (C, linked to the library)."""
    os.makedirs(BINDIR, exist_ok=True)
    common = [os.path.join(HOST, "sbio.c")]
    deps = glob.glob(os.path.join(HOST, "*.[ch]")) + [LIB, os.path.join(INCLUDE, "speckle_b200.h")]
    link = ["-L" + LIBDIR, "-lspeckle_b200", "-Wl,-rpath,$ORIGIN/../lib", "-lm"]
    tools = {"strack": (["track_main.c"], []), "strackw": (["track_main.c"], ["-DSTRACKW"]),
             "cullst": (["cullst_main.c"], [])}
    out = []
    for name, (srcs, defs) in tools.items():
        exe = os.path.join(BINDIR, name)
        if _stale(exe, deps):
            cmd = [CC, "-O2", "-std=gnu11", "-Wall", "-Wno-unused-result"] + defs + \
                [os.path.join(HOST, s) for s in srcs] + common + ["-o", exe] + link
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"building {name} failed:\n{r.stderr}")
        out.append(exe)
    return out


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    build_cli()
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
