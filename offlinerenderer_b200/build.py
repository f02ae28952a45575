"""Builds libwrk.so (the CUDA kernels, the C ABI and the C++ API) in-tree.

    python -m offlinerenderer_b200.build [--force]

All device code is compiled for sm_100a only.  FMA contraction is off
(--fmad=false) so FP32 shading follows the source expression order; kernels
that want FMAs (the BVH slab tests) call fmaf explicitly.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwrk.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
# The system g++ (an exported CXX may be a wrapper without the C++20 headers needed here).
CXX = "g++"

CU_SOURCES = ["bvh_build.cu", "trace.cu", "render.cu", "kernels_misc.cu", "api.cu", "conv_tc.cu", "denoiser.cu", "server.cu"]
CPP_SOURCES = ["wr_api.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "-I", INCLUDE, "-diag-suppress", "550"]
# -fvisibility-inlines-hidden: the inline members of include/wr/*.h (the ones that
# take a Vec3) are compiled into the caller, never exported from libwrk.so.
CXX_FLAGS = ["-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-fvisibility-inlines-hidden", "-I", INCLUDE,
             "-I", os.path.join(CUDA_HOME, "include")]


def _headers():
    out = []
    for d in (CSRC, INCLUDE, os.path.join(INCLUDE, "wr")):
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return out


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
    deps = [os.path.join(CSRC, src)] + _headers()
    if not force and not _stale(obj, deps):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    else:
        cmd = [CXX] + CXX_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles (incrementally) and links libwrk.so; returns its path."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    srcs = CU_SOURCES + CPP_SOURCES
    with cf.ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("linked", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
