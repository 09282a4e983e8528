"""Spectral basis container, its on-disk format, and seeded initial states.

A basis holds everything the per-step hot path reads for one domain
(the reference keeps the same data in ``AbstractSolver``'s members,
Solver/abstractsolver.h:111-126):

* grid: dims, voxel size ``h``, AABB (the tracer's domain box);
* ``active_faces``: reference face ids of the interior faces, the only
  non-zero rows of Phi (``psfsolver.cpp:251-265``);
* ``phi``: ``[n_active][N]`` FP64, ``lam``: ``[N]``, ``gravity``: ``[N]``;
* ``C``: ``[N][N][N]`` FP64, ``C[k][a][j] = advection[k](a, j)``;
* ``sign_bits``: the reference's per-voxel face sign string;
* ``inside``: fluid mask (for seeding particles).

File format ``.psfb`` (little endian): a 256-byte header followed by the
arrays in header order; see :data:`HEADER` and ``include/psf/basis_file.h``.
Any prefix ``N' <= N`` of a basis is again a basis (:meth:`Basis.truncate`).

Compact files ``.psfc`` (header version 2) store Phi as FP32 and leave C out;
loading one promotes Phi to FP64 and rebuilds C from it with the same tensor
builder (FP64 GEMMs, on the GPU when there is one).  The loaded arrays are the
basis: the device path and the oracle consume exactly the same Phi and C.
"""

from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np

from .domain import Domain

MAGIC = b"PSFBASIS"
VERSION = 1
COMPACT_VERSION = 2
# magic, version, dims[3], h, aabb_min[3], aabb_max[3], n_modes, n_faces,
# n_active, n_voxels, n_sign_words, then 7 array offsets (bytes from file start).
HEADER = struct.Struct("<8sI3Id3f3fiqqqq7Q")
HEADER_SIZE = 256
ARRAYS = ("active_faces", "lam", "gravity", "phi", "C", "sign_bits", "inside")


@dataclass
class Basis:
    dims: tuple
    h: float
    aabb_min: np.ndarray
    aabb_max: np.ndarray
    active_faces: np.ndarray  # int32 [n_active]
    lam: np.ndarray  # f64 [N]
    gravity: np.ndarray  # f64 [N]
    phi: np.ndarray  # f64 [n_active, N]
    C: np.ndarray  # f64 [N, N, N]
    sign_bits: np.ndarray  # u32
    inside: np.ndarray  # u8 [V]
    name: str = "basis"

    @property
    def n_modes(self) -> int:
        return int(self.lam.shape[0])

    @property
    def n_active(self) -> int:
        return int(self.active_faces.shape[0])

    @property
    def n_voxels(self) -> int:
        nx, ny, nz = self.dims
        return nx * ny * nz

    @property
    def n_faces(self) -> int:
        nx, ny, nz = self.dims
        return (nz + 1) * nx * ny + (ny + 1) * nx * nz + (nx + 1) * ny * nz

    def truncate(self, n: int) -> "Basis":
        """Exact prefix slice to the lowest ``n`` modes."""
        if n > self.n_modes:
            raise ValueError(f"basis has {self.n_modes} modes, asked for {n}")
        return Basis(
            self.dims, self.h, self.aabb_min, self.aabb_max, self.active_faces,
            self.lam[:n].copy(), self.gravity[:n].copy(),
            np.ascontiguousarray(self.phi[:, :n]), np.ascontiguousarray(self.C[:n, :n, :n]),
            self.sign_bits, self.inside, name=f"{self.name}_n{n}",
        )

    def domain(self) -> Domain:
        nx, ny, nz = self.dims
        return Domain(self.dims, self.h, self.inside.reshape(nz, ny, nx).astype(bool),
                      name=self.name, aabb_min=self.aabb_min, aabb_max=self.aabb_max)

    def phi_full(self) -> np.ndarray:
        full = np.zeros((self.n_faces, self.n_modes))
        full[self.active_faces] = self.phi
        return full

    # ------------------------------------------------------------- file io
    def save(self, path: str, compact: bool = False) -> None:
        """Write a ``.psfb`` file, or with ``compact`` a ``.psfc`` (Phi FP32, no C)."""
        arrays = [
            np.ascontiguousarray(self.active_faces, dtype="<i4"),
            np.ascontiguousarray(self.lam, dtype="<f8"),
            np.ascontiguousarray(self.gravity, dtype="<f8"),
            np.ascontiguousarray(self.phi, dtype="<f4" if compact else "<f8"),
            np.zeros(0, dtype="<f8") if compact else np.ascontiguousarray(self.C, dtype="<f8"),
            np.ascontiguousarray(self.sign_bits, dtype="<u4"),
            np.ascontiguousarray(self.inside, dtype="u1"),
        ]
        offsets, pos = [], HEADER_SIZE
        for a in arrays:
            pos = (pos + 63) // 64 * 64
            offsets.append(pos)
            pos += a.nbytes
        hdr = HEADER.pack(
            MAGIC, COMPACT_VERSION if compact else VERSION, *[int(d) for d in self.dims], float(self.h),
            *[float(v) for v in self.aabb_min], *[float(v) for v in self.aabb_max],
            self.n_modes, self.n_faces, self.n_active, self.n_voxels, int(self.sign_bits.size),
            *offsets,
        )
        tmp = path + ".tmp"
        with open(tmp, "wb") as f:
            f.write(hdr.ljust(HEADER_SIZE, b"\0"))
            for off, a in zip(offsets, arrays):
                f.seek(off)
                f.write(a.tobytes())
        os.replace(tmp, path)

    @staticmethod
    def load(path: str, name: str | None = None, device: str | None = None) -> "Basis":
        with open(path, "rb") as f:
            raw = f.read()
        vals = HEADER.unpack_from(raw, 0)
        if vals[0] != MAGIC or vals[1] not in (VERSION, COMPACT_VERSION):
            raise ValueError(f"{path}: not a basis file")
        compact = vals[1] == COMPACT_VERSION
        dims = tuple(vals[2:5])
        h = vals[5]
        amin = np.array(vals[6:9], dtype=np.float32)
        amax = np.array(vals[9:12], dtype=np.float32)
        N, F, Fa, V, nw = vals[12:17]
        off = vals[17:24]

        def arr(i, dtype, count, shape=None):
            a = np.frombuffer(raw, dtype=dtype, count=count, offset=off[i]).copy()
            return a.reshape(shape) if shape else a

        phi = arr(3, "<f4", Fa * N, (Fa, N)).astype(np.float64) if compact else arr(3, "<f8", Fa * N, (Fa, N))
        b = Basis(
            dims, h, amin, amax,
            arr(0, "<i4", Fa), arr(1, "<f8", N), arr(2, "<f8", N),
            phi, None if compact else arr(4, "<f8", N * N * N, (N, N, N)),
            arr(5, "<u4", nw), arr(6, "u1", V),
            name=name or os.path.splitext(os.path.basename(path))[0],
        )
        if compact:
            b.C = rebuild_tensor(b, device)
        return b


def _cuda_index(device) -> int | None:
    """Device ordinal of a "cuda" / "cuda:K" device string, else None."""
    d = str(device)
    if not d.startswith("cuda"):
        return None
    return int(d.split(":", 1)[1]) if ":" in d else 0


def build_basis(dom: Domain, n_modes: int, device: str = "cpu") -> Basis:
    """Run the per-domain precompute (eigenbasis, curl, gravity, tensor).

    On a CUDA device the whole precompute runs on the GPU
    (:func:`.precompute.build_basis`: Chebyshev-filtered eigen-solve and the
    wedge tensor kernels); on ``"cpu"`` it is the host restatement of
    :mod:`.basis` (SciPy shift-invert ARPACK, FP64 GEMMs).
    """
    from . import basis as B

    idx = _cuda_index(device)
    if idx is not None:
        from . import precompute

        b, _ = precompute.build_basis(dom, n_modes, device=idx)
        return b
    dom.build()
    lam, phi_I = B.eigenbasis(dom, n_modes)
    phi_full = np.zeros((dom.n_faces, n_modes))
    phi_full[dom.interior_faces] = phi_I
    psi = B.curl_basis(dom, phi_full)
    grav = B.gravity_coefficients(dom, phi_full)
    C = B.advection_tensor(dom, phi_full, psi, lam, device=device)
    return Basis(
        dom.dims, dom.h, dom.aabb_min, dom.aabb_max,
        dom.interior_faces.astype(np.int32), lam, grav, phi_I, C,
        dom.sign_bits, dom.inside.ravel().astype(np.uint8), name=dom.name,
    )


def rebuild_tensor(b: Basis, device: str | None = None) -> np.ndarray:
    """C of a basis from its Phi and eigenvalues (the tensor builder of :func:`build_basis`)."""
    from . import basis as B

    if device is None:
        try:
            import torch

            device = "cuda" if torch.cuda.is_available() else "cpu"
        except Exception:
            device = "cpu"
    dom = b.domain()
    dom.build()
    idx = _cuda_index(device)
    if idx is not None:
        from . import precompute

        return precompute.advection_tensor(dom, b.phi, b.lam, device=idx)
    phi_full = b.phi_full()
    psi = B.curl_basis(dom, phi_full)
    return B.advection_tensor(dom, phi_full, psi, b.lam, device=device)


def cached_basis(dom: Domain, n_modes: int, cache_dir: str | None = None,
                 device: str = "cpu") -> Basis:
    """Build a basis once and keep it as ``<cache_dir>/<domain>_n<N>.psfb``."""
    cache_dir = cache_dir or os.environ.get(
        "PSF_BASIS_CACHE", os.path.join(os.path.dirname(os.path.dirname(__file__)), ".basis_cache")
    )
    os.makedirs(cache_dir, exist_ok=True)
    path = os.path.join(cache_dir, f"{dom.name}_n{n_modes}.psfb")
    if os.path.exists(path):
        return Basis.load(path, name=dom.name)
    compact = os.path.join(cache_dir, f"{dom.name}_n{n_modes}.psfc")
    if os.path.exists(compact):
        return Basis.load(compact, name=dom.name, device=None if device == "cpu" else device)
    b = build_basis(dom, n_modes, device=device)
    b.save(path)
    return b


# ------------------------------------------------------------ initial states
def initial_coefficients(n_modes: int, seed: int) -> np.ndarray:
    """``w ~ N(0, 1)`` from ``numpy.random.default_rng(seed)``, scaled to unit energy."""
    w = np.random.default_rng(seed).standard_normal(n_modes)
    return w / np.sqrt(w @ w)


def initial_particles(b: Basis, count: int, seed: int, lifetime: float = np.inf) -> np.ndarray:
    """``count`` particles uniform over the fluid voxels' volume, as float4 (x, y, z, life)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = b.dims
    lo = b.aabb_min.astype(np.float64)
    hi = b.aabb_max.astype(np.float64)
    inside = b.inside.reshape(nz, ny, nx).astype(bool)
    out = np.empty((0, 3))
    while out.shape[0] < count:
        m = max(1024, int(1.3 * (count - out.shape[0])))
        p = lo + rng.random((m, 3)) * (hi - lo)
        g = np.floor((p - lo) / b.h).astype(np.int64)
        g = np.clip(g, 0, np.array([nx - 1, ny - 1, nz - 1]))
        ok = inside[g[:, 2], g[:, 1], g[:, 0]]
        out = np.concatenate([out, p[ok]])
    parts = np.empty((count, 4), dtype=np.float32)
    parts[:, :3] = out[:count]
    parts[:, 3] = np.float32(lifetime)
    return parts
