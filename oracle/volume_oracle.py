"""Test infrastructure (oracle): Python driver for the C restatement of the
reference's particle density volume and ray march (``oracle/psf_volume_oracle.c``,
following Solver/SolverImpl/psfsolvergpu.cpp:876-1022, Resources/Volume/volume.comp
and Resources/Effects/Volume/volume.{vert,frag}).

Only ``tests/`` and ``bench.py``'s CPU baseline leg use this module.

Parity unpinned: the reference renders through OpenGL, which is unavailable
here, its histogram shader is missing from its tree, and it ships no images.
The C restatement is checked against known answers and, pixel by pixel,
against a line-by-line FP32 replay of volume.frag in Python (tests/test_volume.py).
"""

from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "psf_volume_oracle.c")
LIB = os.path.join(HERE, "libpsf_volume_oracle.so")


class View(ct.Structure):
    _fields_ = [
        ("view", ct.c_float * 16),
        ("camera", ct.c_float * 3),
        ("light", ct.c_float * 3),
        ("aabb_min", ct.c_float * 3),
        ("aabb_max", ct.c_float * 3),
        ("width", ct.c_int32),
        ("height", ct.c_int32),
        ("res", ct.c_int32),
    ]


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
        L.psfo_volume_histogram.argtypes = [fp, ct.c_int64, fp, fp, ct.c_int32, ct.POINTER(ct.c_int32)]
        L.psfo_volume_density.argtypes = [ct.POINTER(ct.c_int32), ct.c_int64, ct.c_void_p]
        L.psfo_volume_render.argtypes = [ct.c_void_p, ct.POINTER(View), fp]
        L.psfo_exp_neg_unit.argtypes = [ct.c_float]
        L.psfo_exp_neg_unit.restype = ct.c_float
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def histogram(particles, aabb_min, aabb_max, res: int) -> np.ndarray:
    p = _f(particles).reshape(-1, 4)
    mn, mx = _f(aabb_min), _f(aabb_max)
    h = np.zeros((res, res, res), np.int32)
    lib().psfo_volume_histogram(p.ctypes.data_as(ct.POINTER(ct.c_float)), len(p),
                                mn.ctypes.data_as(ct.POINTER(ct.c_float)), mx.ctypes.data_as(ct.POINTER(ct.c_float)),
                                int(res), h.ctypes.data_as(ct.POINTER(ct.c_int32)))
    return h


def density(hist) -> np.ndarray:
    h = np.ascontiguousarray(hist, dtype=np.int32)
    out = np.zeros(h.shape, np.float16)
    lib().psfo_volume_density(h.ctypes.data_as(ct.POINTER(ct.c_int32)), h.size, out.ctypes.data_as(ct.c_void_p))
    return out


def render(vol, view, aabb_min, aabb_max) -> np.ndarray:
    """rgba float32 (height, width, 4) of an FP16 density (res, res, res)."""
    v = np.ascontiguousarray(vol, dtype=np.float16)
    V = View()
    V.view[:] = [float(x) for x in np.asarray(view["view"], np.float32).reshape(16)]
    V.camera[:] = [float(x) for x in view["camera"]]
    V.light[:] = [float(x) for x in view["light"]]
    V.aabb_min[:] = [float(x) for x in aabb_min]
    V.aabb_max[:] = [float(x) for x in aabb_max]
    V.width, V.height, V.res = int(view["width"]), int(view["height"]), int(v.shape[0])
    out = np.zeros((V.height, V.width, 4), np.float32)
    lib().psfo_volume_render(v.ctypes.data_as(ct.c_void_p), ct.byref(V), out.ctypes.data_as(ct.POINTER(ct.c_float)))
    return out


def exp_neg_unit(y: float) -> float:
    return float(lib().psfo_exp_neg_unit(float(y)))
