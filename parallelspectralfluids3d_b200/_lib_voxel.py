"""ctypes declarations of the mesh voxeliser (``include/psf_voxel.h``)."""

from __future__ import annotations

import ctypes as ct

VOXEL_EXPORTS = (
    "psf_voxel_grid", "psf_voxelizer_create", "psf_voxelizer_destroy", "psf_voxelizer_run",
    "psf_voxelizer_profile", "psf_voxelize",
)


class VoxelMesh(ct.Structure):
    _fields_ = [
        ("vertices", ct.POINTER(ct.c_float)),
        ("n_vertices", ct.c_int64),
        ("triangles", ct.POINTER(ct.c_uint32)),
        ("n_triangles", ct.c_int64),
    ]


def declare(lib) -> None:
    vp = ct.c_void_p
    i32p = ct.POINTER(ct.c_int32)
    fp = ct.POINTER(ct.c_float)
    mp = ct.POINTER(VoxelMesh)
    lib.psf_voxel_grid.argtypes = [mp, ct.c_float, ct.c_int32, i32p, fp]
    lib.psf_voxelizer_create.argtypes = [ct.c_int, ct.c_int64, ct.c_int64, ct.c_int64, ct.POINTER(vp)]
    lib.psf_voxelizer_destroy.argtypes = [vp]
    lib.psf_voxelizer_run.argtypes = [vp, mp, ct.c_float, ct.c_int32, i32p, fp, vp, ct.c_int64]
    lib.psf_voxelizer_profile.argtypes = [vp, ct.c_int32, ct.POINTER(ct.c_double)]
    lib.psf_voxelize.argtypes = [mp, ct.c_float, ct.c_int32, ct.c_int, i32p, fp, vp, ct.c_int64]
