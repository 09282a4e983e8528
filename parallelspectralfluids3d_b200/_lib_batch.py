"""ctypes declarations of the batched engine (``include/psf_batch.h``)."""

from __future__ import annotations

import ctypes as ct

from . import _lib as L

PSF_BATCH_MAX_BASES = 6
PSF_BATCH_MAX_SLOTS = 256

BATCH_EXPORTS = (
    "psf_batch_create", "psf_batch_destroy", "psf_batch_info_get", "psf_batch_set_instance",
    "psf_batch_clear_instance", "psf_batch_step", "psf_batch_sync", "psf_batch_get_stream",
    "psf_batch_get_state", "psf_batch_get_particles", "psf_batch_get_velocity", "psf_batch_get_steps",
    "psf_batch_profile_step", "psf_batch_profile_phases", "psf_batch_device_status", "psf_batch_pool_free",
    "psf_batch_set_instances", "psf_batch_clear_instances", "psf_batch_read_instances",
)


class BatchBasis(ct.Structure):
    _fields_ = [
        ("basis", L.BasisDesc),
        ("slots", ct.c_int32),
        ("max_particles", ct.c_int64),
    ]


class BatchConfig(ct.Structure):
    _fields_ = [
        ("n_bases", ct.c_int32),
        ("bases", ct.POINTER(BatchBasis)),
        ("precision", ct.c_int32),
        ("autotune", ct.c_int32),
        ("gemm_columns", ct.c_int32),
        ("gemm_ctas", ct.c_int32),
        ("particle_pool", ct.c_int64),
        ("contraction_ksplit", ct.c_int32),
        ("unfused", ct.c_int32),
    ]


class InstanceDesc(ct.Structure):
    _fields_ = [
        ("n_modes", ct.c_int32),
        ("params", L.Params),
        ("w0", ct.POINTER(ct.c_double)),
        ("forcing", ct.POINTER(ct.c_double)),
        ("particles", ct.POINTER(ct.c_float)),
        ("n_particles", ct.c_int64),
        ("steps", ct.c_int32),
    ]


class BatchInfo(ct.Structure):
    _fields_ = [
        ("gemm_columns", ct.c_int32),
        ("gemm_ctas", ct.c_int32),
        ("trace_ctas", ct.c_int32),
        ("kernels_per_step", ct.c_int32),
        ("device_bytes", ct.c_int64),
        ("tuned_ms", ct.c_double),
        ("contraction_ksplit", ct.c_int32),
    ]


def declare(lib) -> None:
    """Set argument types of the batch entry points."""
    vp = ct.c_void_p
    i32 = ct.c_int32
    lib.psf_batch_create.argtypes = [ct.POINTER(BatchConfig), ct.c_int, ct.POINTER(vp)]
    lib.psf_batch_destroy.argtypes = [vp]
    lib.psf_batch_info_get.argtypes = [vp, ct.POINTER(BatchInfo)]
    lib.psf_batch_set_instance.argtypes = [vp, i32, i32, ct.POINTER(InstanceDesc)]
    lib.psf_batch_clear_instance.argtypes = [vp, i32, i32]
    lib.psf_batch_step.argtypes = [vp, i32]
    lib.psf_batch_sync.argtypes = [vp]
    lib.psf_batch_get_stream.argtypes = [vp, ct.POINTER(vp)]
    lib.psf_batch_get_state.argtypes = [vp, i32, i32, vp, i32]
    lib.psf_batch_get_particles.argtypes = [vp, i32, i32, vp, ct.c_int64]
    lib.psf_batch_get_velocity.argtypes = [vp, i32, i32, vp, ct.c_int64]
    lib.psf_batch_get_steps.argtypes = [vp, i32, i32, ct.POINTER(ct.c_int64)]
    lib.psf_batch_profile_step.argtypes = [vp, ct.POINTER(ct.c_double), i32]
    lib.psf_batch_profile_phases.argtypes = [vp, ct.POINTER(ct.c_double), i32]
    lib.psf_batch_device_status.argtypes = [vp, ct.POINTER(i32)]
    lib.psf_batch_pool_free.argtypes = [vp, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64)]
    ip = ct.POINTER(i32)
    lib.psf_batch_set_instances.argtypes = [vp, i32, ip, ip, ct.POINTER(ct.POINTER(InstanceDesc)), ip]
    lib.psf_batch_clear_instances.argtypes = [vp, i32, ip, ip]
    lib.psf_batch_read_instances.argtypes = [vp, i32, ip, ip, ct.POINTER(vp), ct.POINTER(vp)]
