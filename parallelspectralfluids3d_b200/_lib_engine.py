"""ctypes declarations of the serving engine (``include/psf_engine.h``)."""

from __future__ import annotations

import ctypes as ct

from . import _lib as L

ENGINE_EXPORTS = (
    "psf_engine_create", "psf_engine_destroy", "psf_engine_submit", "psf_engine_poll", "psf_engine_wait",
    "psf_engine_collect", "psf_engine_drain", "psf_engine_stats_get",
)


class EngineConfig(ct.Structure):
    _fields_ = [
        ("n_bases", ct.c_int32),
        ("bases", ct.POINTER(L.BasisDesc)),
        ("slots", ct.POINTER(ct.c_int32)),
        ("max_particles", ct.c_int64),
        ("particle_pool", ct.c_int64),
        ("hbm_budget_bytes", ct.c_int64),
        ("chunk_steps", ct.c_int32),
        ("autotune", ct.c_int32),
    ]


class Request(ct.Structure):
    _fields_ = [
        ("basis", ct.c_int32),
        ("n_modes", ct.c_int32),
        ("steps", ct.c_int32),
        ("reserved", ct.c_int32),
        ("params", L.Params),
        ("w0", ct.POINTER(ct.c_double)),
        ("forcing", ct.POINTER(ct.c_double)),
        ("particles", ct.POINTER(ct.c_float)),
        ("n_particles", ct.c_int64),
    ]


class RequestInfo(ct.Structure):
    _fields_ = [
        ("id", ct.c_uint64),
        ("status", ct.c_int32),
        ("steps", ct.c_int32),
        ("t_submit", ct.c_double),
        ("t_admit", ct.c_double),
        ("t_done", ct.c_double),
    ]


class EngineStats(ct.Structure):
    _fields_ = [(n, ct.c_int64) for n in (
        "submitted", "admitted", "completed", "queued", "active", "instance_steps", "particle_steps",
        "step_launches", "budget_refusals", "device_bytes", "rollout_bytes")] + [
        (n, ct.c_double) for n in ("t_now", "step_s", "admit_s", "retire_s")]


def declare(lib) -> None:
    vp = ct.c_void_p
    lib.psf_engine_create.argtypes = [ct.POINTER(EngineConfig), ct.c_int, ct.POINTER(vp)]
    lib.psf_engine_destroy.argtypes = [vp]
    lib.psf_engine_submit.argtypes = [vp, ct.POINTER(Request), ct.POINTER(ct.c_uint64)]
    lib.psf_engine_poll.argtypes = [vp, ct.POINTER(ct.c_uint64), ct.c_int32, ct.POINTER(ct.c_int32)]
    lib.psf_engine_wait.argtypes = [vp, ct.c_uint64, ct.c_double]
    lib.psf_engine_collect.argtypes = [vp, ct.c_uint64, vp, ct.c_int32, vp, ct.c_int64, ct.POINTER(RequestInfo)]
    lib.psf_engine_drain.argtypes = [vp, ct.c_double]
    lib.psf_engine_stats_get.argtypes = [vp, ct.POINTER(EngineStats)]
