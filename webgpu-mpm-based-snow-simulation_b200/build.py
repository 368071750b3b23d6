"""In-tree build of libmpm.so for sm_100a.

The kernels are compiled with -fmad=false, IEEE division and square root and
no flush-to-zero: the step's f32 arithmetic follows one fixed operation order
so the fixed-point grid is reproducible bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_PATH = os.path.join(PKG_DIR, "libmpm.so")
SOURCES = ["mpm_kernels.cu", "mpm_mlp.cu", "mpm_splat.cu", "mpm_scatter.cu", "mpm_raymarch.cu", "mpm_mc.cu", "mpm_api.cu", "bvh_build.cpp", "bvh_gpu.cu"]
HEADERS = ["mpm_math.cuh", "mpm_pow_tables.h", "mpm_mc_table.h", "mpm_engine.cuh", "mpm_plast.cuh", "mpm_tc.cuh", "mpm_mlp.cuh",
           os.path.join("..", "..", "include", "mpm.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    for f in SOURCES + HEADERS:
        p = os.path.join(CSRC, f)
        if os.path.exists(p) and os.path.getmtime(p) > t:
            return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile libmpm.so next to this file; returns its path."""
    if not force and not needs_build():
        return LIB_PATH
    cmd = [_nvcc(), *NVCC_FLAGS, "-o", LIB_PATH + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
