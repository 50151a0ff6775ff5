"""Builds the in-tree shared libraries of the package with nvcc for sm_100a.

  libagdeblend.so         AGD_TYPE = float   (agd_deblend, agd_blend, agd_gpu_*)
  libagdeblend_double.so  AGD_TYPE = double

Usage: python -m agdeblend_b200.build [--force] [--ptxas-verbose]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
SOURCES = ["plan.cpp", "engine.cu", "blend.cu", "blend_noalloc.cu", "nn.cu"]
# every header in csrc/ is an input of both libraries (a stale library must
# not travel to the device after a header-only change)
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h")))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIBS = {
    "libagdeblend.so": [],
    "libagdeblend_double.so": ["-DAGD_DOUBLE"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files += [os.path.join(INCLUDE, f) for f in ("agdeblend.h", "agdeblend_gpu.h")]
    return files


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(f) > t for f in _inputs())


def build_lib(name: str, defines, force=False, verbose_ptxas=False) -> str:
    out = os.path.join(PKG, name)
    if not force and not _stale(out):
        return out
    cmd = [nvcc(), "-O3", "-std=c++17", "-lineinfo", *ARCH, "-shared", "-Xcompiler", "-fPIC",
           "-ccbin", "g++", "-I", INCLUDE, "-I", CSRC, *defines,
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", out + ".tmp"]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def build(force: bool = False, verbose_ptxas: bool = False):
    return [build_lib(n, d, force, verbose_ptxas) for n, d in LIBS.items()]


if __name__ == "__main__":
    paths = build(force="--force" in sys.argv, verbose_ptxas="--ptxas-verbose" in sys.argv)
    for p in paths:
        print(p)
