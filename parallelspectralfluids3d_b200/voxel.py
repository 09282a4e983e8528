"""Mesh voxeliser on the GPU: a closed triangle mesh becomes a simulation Domain.

Python face of ``include/psf_voxel.h``.  It replaces ``Model::voxelize``
(Graphics/Model/Model.cpp:203-451), which the reference calls from
``AbstractSolver::setMesh`` (Solver/abstractsolver.cpp:100) to turn a loaded
model into its ``DECMesh3D``.  ``voxelize`` returns the inside flags together
with the grid the reference builds around them (``DECMesh3D(resolution, dims,
resolution, aabb.min)``, Model.cpp:216); ``to_domain`` wraps them as the
``Domain`` the basis builder consumes.

Mesh helpers (``box_mesh``, ``icosphere``, ``torus_mesh``) produce closed,
consistently indexed meshes for tests and benchmarks.
"""

from __future__ import annotations

import ctypes as ct
import math

import numpy as np

from . import _lib as L
from ._lib_voxel import VoxelMesh

REFERENCE = 0
GEOMETRIC = 1
MAX_DIM = 1023


def _mesh(vertices, triangles):
    v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
    m = VoxelMesh(v.ctypes.data_as(ct.POINTER(ct.c_float)), len(v), t.ctypes.data_as(ct.POINTER(ct.c_uint32)), len(t))
    return m, v, t


def grid(vertices, resolution: float, mode: int = REFERENCE):
    """(dims (W, H, D), aabb_min, aabb_max) of a mesh; no device needed."""
    lib = L.load()
    m, _v, _t = _mesh(vertices, np.zeros((0, 3), np.uint32))
    dims = np.zeros(3, np.int32)
    aabb = np.zeros(6, np.float32)
    L.check(lib.psf_voxel_grid(ct.byref(m), float(resolution), int(mode), L.ptr(dims, ct.c_int32),
                               L.ptr(aabb, ct.c_float)))
    return tuple(int(d) for d in dims), aabb[:3].copy(), aabb[3:].copy()


class Voxelizer:
    """Device buffers for meshes and grids up to the given sizes, reused across calls."""

    def __init__(self, max_vertices: int, max_triangles: int, max_voxels: int, device: int = 0):
        self._lib = L.load()
        h = ct.c_void_p()
        L.check(self._lib.psf_voxelizer_create(int(device), int(max_vertices), int(max_triangles), int(max_voxels),
                                               ct.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            self._lib.psf_voxelizer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, vertices, triangles, resolution: float, mode: int = REFERENCE):
        """Inside flags uint8 (D, H, W), dims (W, H, D), aabb_min, aabb_max."""
        m, _v, _t = _mesh(vertices, triangles)
        (W, H, D), _, _ = grid(_v, resolution, mode)
        out = np.empty((D, H, W), np.uint8)
        dims = np.zeros(3, np.int32)
        aabb = np.zeros(6, np.float32)
        L.check(self._lib.psf_voxelizer_run(self._h, ct.byref(m), float(resolution), int(mode),
                                            L.ptr(dims, ct.c_int32), L.ptr(aabb, ct.c_float),
                                            out.ctypes.data_as(ct.c_void_p), out.nbytes))
        return out, (W, H, D), aabb[:3].copy(), aabb[3:].copy()

    def profile(self, iters: int = 10) -> float:
        """Mean device time (ms) of one voxelisation of the last mesh."""
        ms = ct.c_double()
        L.check(self._lib.psf_voxelizer_profile(self._h, int(iters), ct.byref(ms)))
        return ms.value


def voxelize(vertices, triangles, resolution: float, mode: int = REFERENCE, device: int = 0):
    """One-shot: inside flags uint8 (D, H, W), dims (W, H, D), aabb_min, aabb_max."""
    lib = L.load()
    m, v, t = _mesh(vertices, triangles)
    (W, H, D), _, _ = grid(v, resolution, mode)
    out = np.empty((D, H, W), np.uint8)
    dims = np.zeros(3, np.int32)
    aabb = np.zeros(6, np.float32)
    L.check(lib.psf_voxelize(ct.byref(m), float(resolution), int(mode), int(device), L.ptr(dims, ct.c_int32),
                             L.ptr(aabb, ct.c_float), out.ctypes.data_as(ct.c_void_p), out.nbytes))
    return out, (W, H, D), aabb[:3].copy(), aabb[3:].copy()


def to_domain(inside, dims, resolution: float, aabb_min, aabb_max, name: str = "mesh"):
    """The Domain of a voxelised mesh: voxel size = resolution, origin = the model's AABB minimum
    (Model.cpp:216), tracer box = the model's AABB (psfsolver.cpp:80-89)."""
    from .domain import Domain

    return Domain(tuple(dims), float(resolution), np.asarray(inside, dtype=bool), name=name,
                  aabb_min=np.asarray(aabb_min, np.float32), aabb_max=np.asarray(aabb_max, np.float32))


# ------------------------------------------------------------------ meshes
def box_mesh(lo, hi):
    """Closed axis-aligned box (12 triangles, outward winding)."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    v = np.array([[lo[0] if i & 1 == 0 else hi[0], lo[1] if i & 2 == 0 else hi[1], lo[2] if i & 4 == 0 else hi[2]]
                  for i in range(8)], np.float32)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    t = []
    for a, b, c, d in quads:
        t += [(a, b, c), (a, c, d)]
    return v, np.array(t, np.uint32)


def icosphere(subdivisions: int, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    """Closed sphere mesh: an icosahedron with each triangle split in four `subdivisions` times."""
    p = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
             (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(faces, np.int64)
    for _ in range(int(subdivisions)):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01, m12, m20 = (inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base)
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    v = v * float(radius) + np.asarray(center, np.float64)
    return v.astype(np.float32), f.astype(np.uint32)


def torus_mesh(R: float, r: float, nu: int = 48, nv: int = 24):
    """Closed torus around the z axis (major radius R, minor radius r)."""
    u = np.arange(nu) * 2 * np.pi / nu
    w = np.arange(nv) * 2 * np.pi / nv
    U, Wg = np.meshgrid(u, w, indexing="ij")
    x = (R + r * np.cos(Wg)) * np.cos(U)
    y = (R + r * np.cos(Wg)) * np.sin(U)
    z = r * np.sin(Wg)
    v = np.stack([x, y, z], -1).reshape(-1, 3).astype(np.float32)
    idx = lambda i, j: (i % nu) * nv + (j % nv)  # noqa: E731
    t = []
    for i in range(nu):
        for j in range(nv):
            a, b, c, d = idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)
            t += [(a, b, c), (a, c, d)]
    return v, np.array(t, np.uint32)
