"""ctypes binding of ``libpsf_b200.so`` (the C ABI declared in ``include/psf_b200.h``).

There is no fallback: if the CUDA library is missing or fails to load, every
entry point of this package raises.
"""

from __future__ import annotations

import ctypes as ct
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpsf_b200.so")

PSF_OK = 0
PSF_RK1 = 1
PSF_RK4 = 4
PSF_FLAG_RENORM = 1
PSF_FLAG_DECAY_NEG = 2
PSF_FLAG_FORCING = 4
PSF_PRECISION_FP32 = 0
PSF_PRECISION_BF16X2 = 1

ERRORS = {
    -1: "PSF_ERR_INVALID",
    -2: "PSF_ERR_CUDA",
    -3: "PSF_ERR_NOMEM",
    -4: "PSF_ERR_SIGNS",
    -5: "PSF_ERR_STATE",
    -6: "PSF_ERR_UNSUPPORTED",
    -7: "PSF_ERR_TIMEOUT",
}


class PSFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Grid(ct.Structure):
    _fields_ = [
        ("dims", ct.c_uint32 * 3),
        ("resolution", ct.c_double),
        ("aabb_min", ct.c_float * 3),
        ("aabb_max", ct.c_float * 3),
    ]


class BasisDesc(ct.Structure):
    _fields_ = [
        ("grid", Grid),
        ("n_modes", ct.c_int32),
        ("n_active", ct.c_int64),
        ("active_faces", ct.POINTER(ct.c_int32)),
        ("phi", ct.POINTER(ct.c_double)),
        ("advection", ct.POINTER(ct.c_double)),
        ("eigenvalues", ct.POINTER(ct.c_double)),
        ("sign_bits", ct.POINTER(ct.c_uint32)),
    ]


class Params(ct.Structure):
    _fields_ = [
        ("timestep", ct.c_double),
        ("viscosity", ct.c_double),
        ("lifetime", ct.c_float),
        ("integrator", ct.c_int32),
        ("flags", ct.c_uint32),
        ("precision", ct.c_int32),
        ("seed", ct.c_uint64),
    ]


# Symbols declared in include/psf_b200.h (and the batch/engine/no-alloc headers).
EXPORTS = (
    "psf_abi_version", "psf_last_error", "psf_device_count", "psf_create", "psf_destroy",
    "psf_set_params", "psf_set_state", "psf_get_state", "psf_set_forcing", "psf_set_particles",
    "psf_get_particles", "psf_get_velocity", "psf_step", "psf_sync", "psf_get_stream",
    "psf_kernels_per_step", "psf_profile_step", "psf_coeff_step_static",
)

_lib = None


def load(path: str | None = None):
    """Load the CUDA library (raises ``ImportError`` if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing; build it with `python -m parallelspectralfluids3d_b200.build`"
        )
    if path == LIB_PATH:
        from . import build as _build

        if not _build.is_current():
            raise ImportError(f"{path} was not built from the sources beside it; rebuild it with "
                              "`python -m parallelspectralfluids3d_b200.build`")
    L = ct.CDLL(path)
    vp = ct.c_void_p
    L.psf_abi_version.restype = ct.c_int
    L.psf_last_error.restype = ct.c_char_p
    L.psf_device_count.argtypes = [ct.POINTER(ct.c_int)]
    L.psf_create.argtypes = [ct.POINTER(BasisDesc), ct.POINTER(Params), ct.c_int, ct.POINTER(vp)]
    L.psf_destroy.argtypes = [vp]
    L.psf_set_params.argtypes = [vp, ct.POINTER(Params)]
    L.psf_set_state.argtypes = [vp, vp, ct.c_int32]
    L.psf_get_state.argtypes = [vp, vp, ct.c_int32]
    L.psf_set_forcing.argtypes = [vp, vp, ct.c_int32]
    L.psf_set_particles.argtypes = [vp, vp, ct.c_int64]
    L.psf_get_particles.argtypes = [vp, vp, ct.c_int64]
    L.psf_get_velocity.argtypes = [vp, vp, ct.c_int64]
    L.psf_step.argtypes = [vp, ct.c_int32]
    L.psf_sync.argtypes = [vp]
    L.psf_get_stream.argtypes = [vp, ct.POINTER(vp)]
    L.psf_kernels_per_step.argtypes = [vp, ct.POINTER(ct.c_int32)]
    L.psf_profile_step.argtypes = [vp, ct.POINTER(ct.c_double), ct.c_int32]
    L.psf_coeff_step_static.argtypes = [vp, ct.c_int32, vp, vp, vp, ct.POINTER(Params), vp]
    _extend(L)
    _lib = L
    return L


def _extend(L):
    """Declare the batch, engine, voxeliser, volume and precompute entry points."""
    from . import _lib_batch, _lib_engine, _lib_pre, _lib_volume, _lib_voxel

    _lib_batch.declare(L)
    _lib_engine.declare(L)
    _lib_voxel.declare(L)
    _lib_pre.declare(L)
    _lib_volume.declare(L)


def check(rc: int) -> None:
    if rc != PSF_OK:
        msg = load().psf_last_error().decode(errors="replace")
        raise PSFError(rc, msg)


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ct.POINTER(ctype))


def grid_struct(b) -> Grid:
    g = Grid()
    for i in range(3):
        g.dims[i] = int(b.dims[i])
        g.aabb_min[i] = float(b.aabb_min[i])
        g.aabb_max[i] = float(b.aabb_max[i])
    g.resolution = float(b.h)
    return g


class BasisArrays:
    """Keeps the contiguous arrays a :class:`BasisDesc` points at alive."""

    def __init__(self, b):
        self.faces = np.ascontiguousarray(b.active_faces, dtype=np.int32)
        self.phi = np.ascontiguousarray(b.phi, dtype=np.float64)
        self.C = np.ascontiguousarray(b.C, dtype=np.float64)
        self.lam = np.ascontiguousarray(b.lam, dtype=np.float64)
        self.bits = np.ascontiguousarray(b.sign_bits, dtype=np.uint32)
        d = BasisDesc()
        d.grid = grid_struct(b)
        d.n_modes = int(self.lam.shape[0])
        d.n_active = int(self.faces.shape[0])
        d.active_faces = ptr(self.faces, ct.c_int32)
        d.phi = ptr(self.phi, ct.c_double)
        d.advection = ptr(self.C, ct.c_double)
        d.eigenvalues = ptr(self.lam, ct.c_double)
        d.sign_bits = ptr(self.bits, ct.c_uint32)
        self.desc = d


def make_params(dt=0.01, viscosity=0.0, lifetime=np.inf, integrator=PSF_RK4, flags=PSF_FLAG_RENORM,
                precision=PSF_PRECISION_FP32, seed=0) -> Params:
    p = Params()
    p.timestep = float(dt)
    p.viscosity = float(viscosity)
    p.lifetime = float(lifetime)
    p.integrator = int(integrator)
    p.flags = int(flags)
    p.precision = int(precision)
    p.seed = int(seed)
    return p
