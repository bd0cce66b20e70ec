"""Builds the native library in-tree: lithoinv3d_b200/_lib/liblitho_gpu.so.

The library holds the sm_100a kernels, the C ABI (include/litho_gpu.h), the
host model builder and the host L-BFGS driver.  It is compiled with nvcc for
`-gencode arch=compute_100a,code=sm_100a` only.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIBNAME = "liblitho_gpu.so"
SOURCES = ["capi.cu", "noalloc.cu", "mlp.cu", "model_builder.cpp", "lbfgsb.cpp", "surface_io.cpp", "patches.cpp"]
HEADERS = ["kernels_fp64.cuh", "kernels_mixed.cuh", "kernels_facet.cuh", "kernels_patch.cuh", "patches.hpp",
           "kernels_classify.cuh", "mlp_kernels.cuh", "tc_gemm.cuh", "tc_gemm_tma.cuh", "model_builder.hpp",
           "lbfgsb.hpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # FP32 subnormals flushed to zero: rsqrt / reciprocal become one
    # special-function instruction each (no subnormal rescaling).  The FP32
    # far-field values are distances, facet scales and adjoints, all far
    # above 1e-38; FP64 arithmetic is unaffected.
    "-ftz=true",
    "-Xcompiler", "-fPIC", "-shared",
]


def library_path() -> str:
    return os.path.join(LIBDIR, LIBNAME)


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build liblitho_gpu.so")
    return cand


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "litho_gpu.h"))
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    target = library_path()
    if not force and not _stale(target):
        return target
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = target + ".tmp"
    cmd = [_nvcc()] + NVCC_FLAGS + ["-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
