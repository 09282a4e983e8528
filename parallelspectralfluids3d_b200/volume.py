"""Particle density volume and its ray-marched image, on the GPU, headless.

Python face of ``include/psf_volume.h``: the compute part of the reference's
``PSFSolverGPU::drawParticles`` (Solver/SolverImpl/psfsolvergpu.cpp:876-1022) --
particle histogram, FP16 density (Resources/Volume/volume.comp) and the
shadowed emission/absorption ray march of Resources/Effects/Volume/volume.frag --
returning images as arrays instead of drawing into a window.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib as L
from ._lib_volume import VolumeView

RES = 256  # the reference's volume resolution (Solver/abstractsolver.cpp:131-141)


def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """View matrix (glm::lookAt convention, right-handed), as a 4x4 array in column-major order."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, np.asarray(up, np.float64))
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = s, u, -f  # rows of the rotation
    m[0, 3], m[1, 3], m[2, 3] = -s @ eye, -u @ eye, f @ eye
    return m.T.astype(np.float32)  # column-major storage = transpose of the row-major matrix


def make_view(width: int, height: int, eye, target=(0.0, 0.0, 0.0), light=(1.0, 2.0, 1.5), up=(0.0, 1.0, 0.0)):
    """Camera dict accepted by Volume.render and the oracle."""
    return {"view": look_at(eye, target, up), "camera": np.asarray(eye, np.float32),
            "light": np.asarray(light, np.float32), "width": int(width), "height": int(height)}


def _view_struct(view) -> VolumeView:
    V = VolumeView()
    V.view[:] = [float(x) for x in np.asarray(view["view"], np.float32).reshape(16)]
    V.camera[:] = [float(x) for x in view["camera"]]
    V.light[:] = [float(x) for x in view["light"]]
    V.width, V.height = int(view["width"]), int(view["height"])
    return V


class Volume:
    """A res^3 density volume on one device."""

    def __init__(self, res: int = RES, device: int = 0):
        self.lib = L.load()
        self.res = int(res)
        h = ct.c_void_p()
        L.check(self.lib.psf_volume_create(int(device), self.res, ct.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            self.lib.psf_volume_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def splat(self, particles, aabb_min, aabb_max) -> None:
        p = np.ascontiguousarray(particles, dtype=np.float32).reshape(-1, 4)
        mn = np.ascontiguousarray(aabb_min, dtype=np.float32)
        mx = np.ascontiguousarray(aabb_max, dtype=np.float32)
        L.check(self.lib.psf_volume_splat(self._h, p.ctypes.data_as(ct.c_void_p), len(p), L.ptr(mn, ct.c_float),
                                          L.ptr(mx, ct.c_float)))

    def splat_context(self, ctx) -> None:
        """Density of a solver Context's resident particles (no host round trip)."""
        L.check(self.lib.psf_volume_splat_context(self._h, ctx.handle))

    def density(self) -> np.ndarray:
        out = np.empty((self.res,) * 3, np.float16)
        L.check(self.lib.psf_volume_get_density(self._h, out.ctypes.data_as(ct.c_void_p), out.size))
        return out

    def render(self, view) -> np.ndarray:
        """rgba float32 (height, width, 4): light energy and transmittance per pixel."""
        V = _view_struct(view)
        out = np.empty((V.height, V.width, 4), np.float32)
        L.check(self.lib.psf_volume_render(self._h, ct.byref(V), out.ctypes.data_as(ct.c_void_p), out.size))
        return out

    def profile(self, view, iters: int = 10):
        """(splat ms, render ms): mean device times."""
        V = _view_struct(view)
        a, b = ct.c_double(), ct.c_double()
        L.check(self.lib.psf_volume_profile(self._h, ct.byref(V), int(iters), ct.byref(a), ct.byref(b)))
        return a.value, b.value


def write_ppm(path: str, rgba: np.ndarray) -> None:
    """8-bit binary PPM of an image's light energy (top row first)."""
    img = np.clip(rgba[::-1, :, :3], 0.0, 1.0)
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(f"P6 {w} {h} 255\n".encode())
        f.write((img * 255.0 + 0.5).astype(np.uint8).tobytes())
