"""Builds the native library ``zigtrace_b200/libzt_b200.so`` in-tree.

Host C++ is compiled with g++ and the CUDA sources with nvcc for sm_100a
only, both with floating-point contraction off (``-ffp-contract=off`` /
``-fmad=false``): the renderer's f64 arithmetic must round exactly as the
reference's strict-float Zig code.  Rebuilds only what is out of date.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libzt_b200.so"

NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
            f"-I{INCLUDE}", f"-I{CSRC}"]
NVCCFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xptxas", "-v", "-Xcompiler",
             "-fPIC,-ffp-contract=off,-fno-fast-math", f"-I{INCLUDE}", f"-I{CSRC}", *ARCH]

CPP_SOURCES = ["scene_host.cpp"]
CU_SOURCES = ["render.cu", "output.cu", "bvh_build.cu"]
HEADERS = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "zigtrace_b200.h"]


def _newest(paths):
    return max(p.stat().st_mtime for p in paths if p.exists())


def _run(cmd, log=None):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.write_text(res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build command failed: {' '.join(cmd)}")
    return res


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the native library if any source is newer than it."""
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build zigtrace_b200")
    BUILD.mkdir(exist_ok=True)
    hdr_time = _newest(HEADERS)
    objects = []
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objects.append(o)
        if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hdr_time):
            _run([CXX, *CXXFLAGS, "-c", str(s), "-o", str(o)])
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objects.append(o)
        if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hdr_time):
            res = _run([NVCC, *NVCCFLAGS, "-c", str(s), "-o", str(o)], log=BUILD / (src + ".ptxas.txt"))
            if verbose:
                print(res.stderr)
    if force or not LIB.exists() or LIB.stat().st_mtime < _newest(objects):
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objects)])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
