"""Build ``libpsf_b200.so`` (CUDA kernels for sm_100a + C ABI + C++ solver) in-tree.

The library is compiled with nvcc for ``sm_100a`` only; nothing is JIT-built
at import time.  ``python -m parallelspectralfluids3d_b200.build`` rebuilds.
"""

from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libpsf_b200.so")
TOOL = os.path.join(PKG, "psf_run")

CU_SOURCES = ["psf_b200.cu", "psf_batch.cu", "psf_noalloc.cu", "psf_voxel.cu", "psf_volume.cu"]
CPP_SOURCES = ["psf_api.cpp", "psf_batch_api.cpp", "abstractsolver.cpp", "psfsolvercuda.cpp",
               "basis_file.cpp", "psf_engine.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _sources():
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES + CPP_SOURCES]
    return [s for s in srcs if os.path.exists(s)]


def _stale(target, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = _sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    headers += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    headers += [os.path.join(INCLUDE, "psf", f) for f in os.listdir(os.path.join(INCLUDE, "psf"))]
    if force or _stale(LIB, srcs + headers):
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
               "-shared", "-I", INCLUDE, "-I", CSRC, "-o", LIB, *srcs, "-lcudart", "-lpthread"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    tool_src = os.path.join(CSRC, "psf_run.cpp")
    if os.path.exists(tool_src) and (force or _stale(TOOL, [tool_src, LIB])):
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, "-o", TOOL, tool_src, "-L", PKG,
               "-lpsf_b200", f"-Wl,-rpath,{PKG}", "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
