"""Builds libfpb200.so (the sm_100a CUDA library behind include/fp_capi.h) and libfocalors_b200.so (the
C++ drop-in interface of focalors_poisson_b200/cpp/ over it) in-tree.

    python -m focalors_poisson_b200.build [--cases <reference case dir>]

Compiles every csrc/*.cu with nvcc for sm_100a (-gencode arch=compute_100a,code=sm_100a) into
focalors_poisson_b200/_build/ and links focalors_poisson_b200/libfpb200.so; compiles cpp/fp_host.cpp and
cpp/fp_host3d.cpp with g++ into focalors_poisson_b200/libfocalors_b200.so. With --cases, also compiles the reference's own 2D
validation drivers (poisson_solver_reference.cpp, concat_solver_reference.cpp), unchanged, against the
drop-in headers into focalors_poisson_b200/_build/cases/. Rebuilds only what changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libfpb200.so")
CPP = os.path.join(PKG, "cpp")
DROPIN_LIB = os.path.join(PKG, "libfocalors_b200.so")
CASES = os.path.join(BUILD, "cases")
# The reference's 2D validation drivers that use only the serial solver interface.
REFERENCE_DRIVERS = ("poisson_solver_reference", "concat_solver_reference")
GXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-I" + CPP, "-I" + os.path.join(ROOT, "include")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _newest_header() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, extra=()) -> str:
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return obj
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build_library(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(_compile, srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcublas", "-lcusolver"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


def gxx() -> str:
    for cand in (shutil.which("g++"), "/usr/bin/g++"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("g++ not found")


def _newer(target: str, deps) -> bool:
    return os.path.exists(target) and os.path.getmtime(target) >= max(os.path.getmtime(d) for d in deps)


def _run(cmd, what):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{what} failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_dropin(verbose: bool = False) -> str:
    """libfocalors_b200.so: Geometry2D / Variable2D / PoissonSolver2D / ConcatPoissonSolver2D and their 3D
    counterparts over libfpb200."""
    build_library()
    srcs = [os.path.join(CPP, "fp_host.cpp"), os.path.join(CPP, "fp_host3d.cpp")]
    deps = srcs + [LIB] + glob.glob(os.path.join(CPP, "**", "*.h*"), recursive=True)
    if not _newer(DROPIN_LIB, deps):
        _run([gxx()] + GXX_FLAGS + ["-shared"] + srcs + ["-o", DROPIN_LIB, "-L" + PKG, "-lfpb200",
                                    "-Wl,-rpath,$ORIGIN"], "g++ (libfocalors_b200.so)")
    if verbose:
        print(DROPIN_LIB)
    return DROPIN_LIB


def compile_driver(src: str, out: str) -> str:
    """Compiles one C++ case driver against the drop-in headers and links it to libfocalors_b200.so."""
    build_dropin()
    deps = [src, DROPIN_LIB] + glob.glob(os.path.join(CPP, "**", "*.h*"), recursive=True)
    if not _newer(out, deps):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        rpath = os.path.relpath(PKG, os.path.dirname(os.path.abspath(out)))
        _run([gxx()] + GXX_FLAGS + [src, "-o", out, "-L" + PKG, "-lfocalors_b200", "-lfpb200",
                                    "-Wl,-rpath,$ORIGIN/" + rpath], f"g++ ({os.path.basename(src)})")
    return out


def build_reference_drivers(case_dir: str) -> list:
    """The reference's validation drivers, compiled from its own files without change."""
    return [compile_driver(os.path.join(case_dir, n + ".cpp"), os.path.join(CASES, n)) for n in REFERENCE_DRIVERS]


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", default=None, help="directory holding the reference's 2D validation drivers")
    a = ap.parse_args()
    build_library(verbose=True)
    build_dropin(verbose=True)
    if a.cases:
        for p in build_reference_drivers(a.cases):
            print(p)
