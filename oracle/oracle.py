"""Test infrastructure (oracle): Python driver for the FP64 C restatement.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
legs use this module.  It builds ``oracle/libpsf_oracle.so`` from
``oracle/psf_oracle.c`` and runs the reference's step semantics
(Solver/SolverImpl/psfsolver.cpp:21-234) on a basis.

Parity unpinned: the reference has no tests or golden vectors for this path
and does not build here (Eigen3, glm, OpenCL, Qt absent).
"""

from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "psf_oracle.c")
LIB = os.path.join(HERE, "libpsf_oracle.so")

FLAG_RENORM = 1
FLAG_DECAY_NEG = 2
FLAG_FORCING = 4


class Grid(ct.Structure):
    _fields_ = [
        ("dims", ct.c_uint32 * 3),
        ("h", ct.c_double),
        ("aabb_min", ct.c_float * 3),
        ("aabb_max", ct.c_float * 3),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle (portable x86-64-v3 code, OpenMP)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"]
        subprocess.run(cmd, check=True)
    from . import volume_oracle, voxel_oracle

    voxel_oracle.build(force)
    volume_oracle.build(force)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ct.CDLL(LIB)
        dp = ct.POINTER(ct.c_double)
        fp = ct.POINTER(ct.c_float)
        L.psfo_coeff_step.argtypes = [ct.c_int32, dp, dp, dp, ct.c_double, ct.c_double, ct.c_uint32, dp, dp]
        L.psfo_contract.argtypes = [ct.c_int32, dp, dp, dp]
        L.psfo_reconstruct.argtypes = [ct.c_int64, ct.c_int32, dp, ct.POINTER(ct.c_int32), ct.c_int64, dp, fp]
        L.psfo_trace.argtypes = [ct.POINTER(Grid), fp, ct.POINTER(ct.c_uint32), dp, fp, ct.c_int64,
                                 ct.c_double, ct.c_int32, ct.c_float, ct.c_uint64, ct.c_uint64]
        L.psfo_hash.argtypes = [ct.c_uint64, ct.c_uint64, ct.c_uint32, ct.c_uint32]
        L.psfo_hash.restype = ct.c_uint32
        L.psfo_num_threads.restype = ct.c_int
        L.psfo_set_threads.argtypes = [ct.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ct.POINTER(t))


def grid_of(b) -> Grid:
    g = Grid()
    for i in range(3):
        g.dims[i] = int(b.dims[i])
        g.aabb_min[i] = float(b.aabb_min[i])
        g.aabb_max[i] = float(b.aabb_max[i])
    g.h = float(b.h)
    return g


def num_threads() -> int:
    return int(lib().psfo_num_threads())


def set_threads(n: int) -> None:
    lib().psfo_set_threads(int(n))


def contract(C: np.ndarray, w: np.ndarray) -> np.ndarray:
    N = w.shape[0]
    C = np.ascontiguousarray(C, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    dw = np.empty(N)
    lib().psfo_contract(N, _p(C, ct.c_double), _p(w, ct.c_double), _p(dw, ct.c_double))
    return dw


class OracleRollout:
    """FP64 reference-semantics rollout of one instance on a basis."""

    def __init__(self, b, w0, particles=None, dt=0.01, viscosity=0.0, flags=FLAG_RENORM,
                 integrator=1, lifetime=np.inf, seed=0, forcing=None, reconstruct=True, positions="f64"):
        self.b = b
        self.N = b.n_modes
        self.C = np.ascontiguousarray(b.C, dtype=np.float64)
        self.lam = np.ascontiguousarray(b.lam, dtype=np.float64)
        self.phi = np.ascontiguousarray(b.phi, dtype=np.float64)
        self.faces = np.ascontiguousarray(b.active_faces, dtype=np.int32)
        self.bits = np.ascontiguousarray(b.sign_bits, dtype=np.uint32)
        self.force = None if forcing is None else np.ascontiguousarray(forcing, dtype=np.float64)
        if self.force is not None:
            flags |= FLAG_FORCING
        self.flags = flags
        self.dt = float(dt)
        self.visc = float(viscosity)
        self.integrator = int(integrator)
        self.lifetime = float(lifetime)
        self.seed = int(seed)
        self.w = np.array(w0, dtype=np.float64)
        self.dw = np.zeros(self.N)
        self.u = np.zeros(b.n_faces, dtype=np.float32)
        self.grid = grid_of(b)
        self.step_index = 0
        self.reconstruct = bool(reconstruct)
        # "f64": positions carried in FP64 (the ground truth).  "f32": rounded to
        # FP32 after every step, as the reference stores them (glm::vec4,
        # Graphics/Particle/Particle.h:14; psfsolver.cpp:215).
        if positions not in ("f64", "f32"):
            raise ValueError("positions must be 'f64' or 'f32'")
        self.positions = positions
        if particles is None:
            particles = np.zeros((0, 4), dtype=np.float32)
        particles = np.asarray(particles, dtype=np.float32)
        self.pos = np.ascontiguousarray(particles[:, :3], dtype=np.float64)
        self.life = np.ascontiguousarray(particles[:, 3], dtype=np.float32)

    def coeff_step(self):
        L = lib()
        fp = _p(self.force, ct.c_double) if self.force is not None else None
        L.psfo_coeff_step(self.N, _p(self.C, ct.c_double), _p(self.lam, ct.c_double), fp, self.dt,
                          self.visc, self.flags, _p(self.w, ct.c_double), _p(self.dw, ct.c_double))
        if not self.reconstruct:
            return
        L.psfo_reconstruct(self.phi.shape[0], self.N, _p(self.phi, ct.c_double),
                           _p(self.faces, ct.c_int32), self.u.shape[0], _p(self.w, ct.c_double),
                           _p(self.u, ct.c_float))

    def trace(self):
        P = self.pos.shape[0]
        if P:
            lib().psfo_trace(ct.byref(self.grid), _p(self.u, ct.c_float), _p(self.bits, ct.c_uint32),
                             _p(self.pos, ct.c_double), _p(self.life, ct.c_float), P, self.dt,
                             self.integrator, self.lifetime, self.seed, self.step_index)

    def step(self, n: int = 1):
        for _ in range(n):
            self.coeff_step()
            self.trace()
            if self.positions == "f32":
                self.pos[...] = self.pos.astype(np.float32)
            self.step_index += 1
        return self

    def particles(self) -> np.ndarray:
        out = np.empty((self.pos.shape[0], 4), dtype=np.float32)
        out[:, :3] = self.pos
        out[:, 3] = self.life
        return out
