"""Build recipe of the in-tree B200 library `unblending_b200/libunblending.so.1`.

Each CUDA translation unit is compiled for sm_100a with nvcc; the host C++
with g++; the shared object is linked with the exported-symbol list of
csrc/exports.map and soname libunblending.so.1 (the reference's SDK naming,
unblending/CMakeLists.txt:43-56). Objects are rebuilt only when a source or
header is newer. Usage: `python unblending_b200/build.py [--force]` (by path: importing the
package needs the library this produces).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libunblending.so.1")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]

# (source, extra nvcc flags). The solver (one unit per layer count) and the
# filter keep IEEE multiply/add rounding (no FMA contraction) like the
# reference's CUDA build.
UNITS = [
    *[(f"solver_l{L}.cu", ["--fmad=false"]) for L in range(1, 9)],
    ("solver_launch.cu", []),
    ("filter.cu", ["--fmad=false"]),
    ("noalloc.cu", []),
    ("order.cu", []),
    ("mlp.cu", []),
    ("mlp_data.cu", []),
    ("pixels.cpp", ["-I" + os.path.join(ROOT, "include")]),
    ("layer_infos.cpp", ["-I" + os.path.join(ROOT, "include")]),
    ("unblending_c.cpp", []),
]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h")) + glob.glob(os.path.join(ROOT, "include", "unblending", "*.hpp"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, flags, verbose):
    out = os.path.join(BUILD, os.path.basename(src) + ".o")
    path = os.path.join(CSRC, src)
    if not _stale(out, [path] + _headers()):
        return out
    if src.endswith(".cu"):
        cmd = [NVCC, *ARCH, *COMMON, *flags, "-c", path, "-o", out]
    else:
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-I" + os.path.join(CUDA, "include"),
               "-I" + os.path.join(ROOT, "include"), *flags, "-c", path, "-o", out]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return out


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in glob.glob(os.path.join(BUILD, "*.o")):
            os.remove(f)
    units = [(s, f) for s, f in UNITS if os.path.exists(os.path.join(CSRC, s))]
    with cf.ThreadPoolExecutor(max_workers=len(units)) as ex:
        objs = list(ex.map(lambda u: _compile(u[0], u[1], verbose), units))
    if _stale(LIB, objs + [os.path.join(CSRC, "exports.map")]):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xlinker", "-soname=libunblending.so.1",
               "-Xlinker", "--version-script=" + os.path.join(CSRC, "exports.map"), "-lcudart", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    link = os.path.join(HERE, "libunblending.so")
    if not os.path.islink(link) or os.readlink(link) != "libunblending.so.1":
        if os.path.lexists(link):
            os.remove(link)
        os.symlink("libunblending.so.1", link)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
