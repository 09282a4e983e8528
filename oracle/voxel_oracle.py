"""Test infrastructure (oracle): Python driver for the C restatement of the
reference's slice-map mesh voxeliser (``oracle/psf_voxel_oracle.c``, following
Graphics/Model/Model.cpp:203-451 and Resources/Voxel/voxel.{vert,geom,frag}).

Only ``tests/`` and ``bench.py``'s CPU baseline leg use this module.

Parity unpinned: the reference voxelises through OpenGL, which is unavailable
here, and ships no voxelised fixtures; the restatement fixes GL's
implementation-defined rasterisation rules (1/256-pixel snapping, exact edge
functions, a down-or-right edge ownership rule) and is checked against
known answers instead (axis-aligned boxes, spheres, watertightness) and
against a literal Python replay of the shader's bit loops and of the
read-back loops (tests/test_voxel.py).
"""

from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "psf_voxel_oracle.c")
LIB = os.path.join(HERE, "libpsf_voxel_oracle.so")

REFERENCE = 0
GEOMETRIC = 1


def build(force: bool = False) -> str:
    """Compile with floating-point contraction off, so every rounding step is the written one."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"]
        subprocess.run(cmd, check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ct.CDLL(LIB)
        fp = ct.POINTER(ct.c_float)
        L.psfo_voxel_dims.argtypes = [fp, ct.c_int64, ct.c_float, ct.c_int, ct.POINTER(ct.c_int32), fp]
        L.psfo_voxelize.argtypes = [fp, ct.c_int64, ct.POINTER(ct.c_uint32), ct.c_int64, ct.c_float, ct.c_int,
                                    ct.POINTER(ct.c_uint8)]
        _lib = L
    return _lib


def grid(vertices, resolution, mode=REFERENCE):
    """(dims (W, H, D), aabb_min, aabb_max) of a mesh, or ValueError."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
    dims = np.zeros(3, np.int32)
    aabb = np.zeros(6, np.float32)
    rc = lib().psfo_voxel_dims(v.ctypes.data_as(ct.POINTER(ct.c_float)), len(v), float(resolution), int(mode),
                               dims.ctypes.data_as(ct.POINTER(ct.c_int32)), aabb.ctypes.data_as(ct.POINTER(ct.c_float)))
    if rc != 0:
        raise ValueError("mesh does not voxelise at this resolution")
    return tuple(int(d) for d in dims), aabb[:3].copy(), aabb[3:].copy()


def voxelize(vertices, triangles, resolution, mode=REFERENCE) -> np.ndarray:
    """Inside flags, uint8 of shape (D, H, W) (voxel id z*W*H + y*W + x)."""
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
    (W, H, D), _, _ = grid(v, resolution, mode)
    out = np.zeros((D, H, W), np.uint8)
    rc = lib().psfo_voxelize(v.ctypes.data_as(ct.POINTER(ct.c_float)), len(v),
                             t.ctypes.data_as(ct.POINTER(ct.c_uint32)), len(t), float(resolution), int(mode),
                             out.ctypes.data_as(ct.POINTER(ct.c_uint8)))
    if rc != 0:
        raise ValueError("bad mesh (triangle index out of range)")
    return out
