"""Build ``libpsf_b200.so`` (CUDA kernels for sm_100a + C ABI + C++ solver) in-tree.

The library is compiled with nvcc for ``sm_100a`` only; nothing is JIT-built
at import time.  ``python -m parallelspectralfluids3d_b200.build`` rebuilds.

Staleness is decided by content, not by file times: the SHA-256 of every
source and header plus the compiler command is written next to the library
(``libpsf_b200.so.stamp``) after a successful build, and a build whose digest
differs from the stamp recompiles.  ``_lib.load`` refuses a library whose
stamp does not match the sources beside it, so a copied tree can never run a
library built from other sources.
"""

from __future__ import annotations

import hashlib
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libpsf_b200.so")
TOOL = os.path.join(PKG, "psf_run")

CU_SOURCES = ["psf_b200.cu", "psf_batch.cu", "psf_noalloc.cu", "psf_voxel.cu", "psf_volume.cu",
              "psf_precompute.cu"]
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


STAMP = LIB + ".stamp"
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-shared"]
LIBS = ["-lcudart", "-lpthread"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    hs += [os.path.join(INCLUDE, "psf", f) for f in os.listdir(os.path.join(INCLUDE, "psf"))]
    return sorted(hs)


def source_digest() -> str:
    """SHA-256 over the library's sources, headers and compiler flags."""
    h = hashlib.sha256()
    h.update(" ".join(ARCH + FLAGS + LIBS + CU_SOURCES + CPP_SOURCES).encode())
    for f in _sources() + _headers():
        h.update(os.path.relpath(f, ROOT).encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def built_digest() -> str | None:
    """The digest the present library was built from (None if unknown)."""
    if not (os.path.exists(LIB) and os.path.exists(STAMP)):
        return None
    with open(STAMP) as f:
        return f.read().strip() or None


def is_current() -> bool:
    return built_digest() == source_digest()


def _stale(target, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


last_build_compiled = False


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library unless its stamp matches the sources; sets ``last_build_compiled``."""
    global last_build_compiled
    srcs = _sources()
    digest = source_digest()
    last_build_compiled = False
    if force or built_digest() != digest:
        cmd = [nvcc(), *ARCH, *FLAGS, "-I", INCLUDE, "-I", CSRC, "-o", LIB, *srcs, *LIBS]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        if os.path.exists(STAMP):
            os.unlink(STAMP)
        subprocess.run(cmd, check=True)
        with open(STAMP, "w") as f:
            f.write(digest + "\n")
        last_build_compiled = True
    tool_src = os.path.join(CSRC, "psf_run.cpp")
    if os.path.exists(tool_src) and (force or _stale(TOOL, [tool_src, LIB])):
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, "-o", TOOL, tool_src, "-L", PKG,
               "-lpsf_b200", f"-Wl,-rpath,{PKG}", "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
