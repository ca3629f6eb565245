"""Builds the sm_100a shared library ``libmpm_b200.so`` in-tree.

Usage: ``python -m mpm_cuda_b200.build`` (or ``build()`` from Python).
The library exports the C ABI declared in ``include/mpm_b200.h``.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libmpm_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE]
CU_SOURCES = ["mpm_abi.cu", "mpm_engine.cu", "mpm_fused_plain.cu", "mpm_fused_fixed.cu", "mpm_fused_paged.cu",
              "mpm_fused_paged_fixed.cu", "mpm_fused_sur.cu", "mpm_noalloc.cu", "mpm_surrogate.cu", "mpm_seed.cu"]
CPP_SOURCES = ["bgeo.cpp"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libmpm_b200.so")
    return cand


def _newest_source_mtime() -> float:
    t = 0.0
    for d in (CSRC, INCLUDE):
        for name in os.listdir(d):
            t = max(t, os.path.getmtime(os.path.join(d, name)))
    return max(t, os.path.getmtime(__file__))


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compiles every source for sm_100a and links ``libmpm_b200.so``."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_source_mtime():
        return LIB
    nvcc = _nvcc()
    os.makedirs(BUILD_DIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []

    def compile_one(src: str) -> str:
        obj = os.path.join(BUILD_DIR, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cxx = shutil.which("g++") or "g++"
            cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-I", CSRC, "-I", INCLUDE, "-c",
                   os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if ptxas_info or verbose:
            sys.stderr.write(r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        return obj

    # the translation units are independent: compile them in parallel
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objs = list(pool.map(compile_one, CU_SOURCES + CPP_SOURCES))
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
