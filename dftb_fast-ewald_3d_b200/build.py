"""Build libewald_b200.so in-tree with nvcc for sm_100a.

Usage: python build.py [--force] [--verbose]   (or ewald_b200.build() from Python)

Each translation unit is compiled to an object under _build/ (skipped when the
object is newer than its sources and headers), then linked into
libewald_b200.so next to this file, so that the library travels with the
source tree.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libewald_b200.so")

SOURCES = ["ewg_chain.cpp", "ewg_real.cu", "ewg_mesh.cu", "ewg_stencil.cu", "ewg_api.cu",
           "ewg_static.cu", "ewg_external.cu", "ewg_points.cu"]
HEADERS = ["ewg_internal.h", "ewg_kernels.h", "ewg_fft.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # The image's CXX wrapper lacks some runtime specs; the system g++ is used.
    return shutil.which("g++") or "g++"


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "ewald_b200.h")]
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", host_cxx(),
              "-I", os.path.join(ROOT, "include")]
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [path, __file__] + headers):
            continue
        if src.endswith(".cu"):
            cmd = [nvcc()] + common + ["-c", path, "-o", obj] + ARCH + ["-lineinfo", "--expt-relaxed-constexpr"]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
        else:
            cmd = [host_cxx(), "-O3", "-std=c++17", "-fPIC", "-I", os.path.join(ROOT, "include"),
                   "-I", "/usr/local/cuda/include", "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-ccbin", host_cxx()] + ARCH + objs + ["-o", LIB, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/smem usage")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))
    sys.exit(0)
