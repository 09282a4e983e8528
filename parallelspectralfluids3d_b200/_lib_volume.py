"""ctypes declarations of the particle density volume (``include/psf_volume.h``)."""

from __future__ import annotations

import ctypes as ct

VOLUME_EXPORTS = (
    "psf_volume_create", "psf_volume_destroy", "psf_volume_splat", "psf_volume_splat_context",
    "psf_volume_get_density", "psf_volume_render", "psf_volume_profile",
)


class VolumeView(ct.Structure):
    _fields_ = [
        ("view", ct.c_float * 16),
        ("camera", ct.c_float * 3),
        ("light", ct.c_float * 3),
        ("width", ct.c_int32),
        ("height", ct.c_int32),
    ]


def declare(lib) -> None:
    vp = ct.c_void_p
    fp = ct.POINTER(ct.c_float)
    vv = ct.POINTER(VolumeView)
    lib.psf_volume_create.argtypes = [ct.c_int, ct.c_int32, ct.POINTER(vp)]
    lib.psf_volume_destroy.argtypes = [vp]
    lib.psf_volume_splat.argtypes = [vp, vp, ct.c_int64, fp, fp]
    lib.psf_volume_splat_context.argtypes = [vp, vp]
    lib.psf_volume_get_density.argtypes = [vp, vp, ct.c_int64]
    lib.psf_volume_render.argtypes = [vp, vv, vp, ct.c_int64]
    lib.psf_volume_profile.argtypes = [vp, vv, ct.c_int32, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)]
