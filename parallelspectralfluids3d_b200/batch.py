"""Python host side of the batched engine (``include/psf_batch.h``).

A :class:`Batch` holds one or more domain bases, each with a number of
instance slots.  Every occupied slot is one rollout of the reference's
per-step update (Solver/SolverImpl/psfsolver.cpp:21-234) with its own mode
count (a prefix of its basis), time step, flags, forcing, state and
particles; one :meth:`Batch.step` advances all of them on the tensor cores.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib as L
from . import _lib_batch as LB


class Batch:
    """Slots of one or more bases stepped together (BF16 hi/lo tensor-core path)."""

    def __init__(self, bases, slots, max_particles, device: int = 0, autotune: bool = True,
                 gemm_columns: int = 0, gemm_ctas: int = 0, particle_pool: int = 0, ksplit: int = 0,
                 fused: bool = True):
        """``bases``: list of :class:`~.fixture.Basis`; ``slots`` / ``max_particles``: per basis (int or list)."""
        self.lib = L.load()
        n = len(bases)
        slots = [int(slots)] * n if np.isscalar(slots) else [int(s) for s in slots]
        max_particles = ([int(max_particles)] * n if np.isscalar(max_particles)
                         else [int(p) for p in max_particles])
        self.bases = list(bases)
        self.slots = slots
        self.max_particles = max_particles
        self._arrays = [L.BasisArrays(b) for b in bases]
        arr = (LB.BatchBasis * n)()
        for i, a in enumerate(self._arrays):
            arr[i].basis = a.desc
            arr[i].slots = slots[i]
            arr[i].max_particles = max_particles[i]
        cfg = LB.BatchConfig()
        cfg.n_bases = n
        cfg.bases = arr
        cfg.precision = L.PSF_PRECISION_BF16X2
        cfg.autotune = 1 if autotune else 0
        cfg.gemm_columns = int(gemm_columns)
        cfg.gemm_ctas = int(gemm_ctas)
        cfg.particle_pool = int(particle_pool)
        cfg.contraction_ksplit = int(ksplit)
        cfg.unfused = 0 if fused else 1
        self.handle = ct.c_void_p()
        L.check(self.lib.psf_batch_create(ct.byref(cfg), int(device), ct.byref(self.handle)))
        self._n_modes = {}
        self._n_particles = {}

    def close(self) -> None:
        if self.handle:
            L.check(self.lib.psf_batch_destroy(self.handle))
            self.handle = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------- instances
    def set_instance(self, basis: int, slot: int, w0, params: L.Params, particles=None, forcing=None,
                     n_modes: int | None = None, steps: int = 0) -> None:
        """Place a rollout in a slot; ``steps > 0`` stops it after that many steps."""
        w0 = np.ascontiguousarray(w0, dtype=np.float64)
        n = int(n_modes if n_modes is not None else w0.shape[0])
        d = LB.InstanceDesc()
        d.n_modes = n
        d.params = params
        d.w0 = L.ptr(w0, ct.c_double)
        keep = [w0]
        if forcing is not None:
            f = np.ascontiguousarray(forcing, dtype=np.float64)
            keep.append(f)
            d.forcing = L.ptr(f, ct.c_double)
        P = 0
        if particles is not None:
            p = np.ascontiguousarray(particles, dtype=np.float32).reshape(-1, 4)
            keep.append(p)
            P = int(p.shape[0])
            if P:
                d.particles = L.ptr(p, ct.c_float)
        d.n_particles = P
        d.steps = int(steps)
        L.check(self.lib.psf_batch_set_instance(self.handle, int(basis), int(slot), ct.byref(d)))
        self._n_modes[(basis, slot)] = n
        self._n_particles[(basis, slot)] = P

    def set_instances(self, items) -> np.ndarray:
        """Place many rollouts with one synchronisation; ``items`` holds dicts with the keys of
        ``set_instance`` (basis, slot, w0, params, particles, forcing, n_modes, steps).  Returns each
        placement's status (0 or a PSF_ERR_* code)."""
        n = len(items)
        descs = (LB.InstanceDesc * n)()
        ptrs = (ct.POINTER(LB.InstanceDesc) * n)()
        basis = np.zeros(n, np.int32)
        slot = np.zeros(n, np.int32)
        keep = []
        for i, it in enumerate(items):
            w0 = np.ascontiguousarray(it["w0"], dtype=np.float64)
            keep.append(w0)
            d = descs[i]
            d.n_modes = int(it.get("n_modes") or w0.shape[0])
            d.params = it["params"]
            d.w0 = L.ptr(w0, ct.c_double)
            if it.get("forcing") is not None:
                f = np.ascontiguousarray(it["forcing"], dtype=np.float64)
                keep.append(f)
                d.forcing = L.ptr(f, ct.c_double)
            P = 0
            if it.get("particles") is not None:
                p = np.ascontiguousarray(it["particles"], dtype=np.float32).reshape(-1, 4)
                keep.append(p)
                P = int(p.shape[0])
                if P:
                    d.particles = L.ptr(p, ct.c_float)
            d.n_particles = P
            d.steps = int(it.get("steps", 0))
            ptrs[i] = ct.pointer(d)
            basis[i], slot[i] = int(it["basis"]), int(it["slot"])
        status = np.zeros(n, np.int32)
        L.check(self.lib.psf_batch_set_instances(self.handle, n, L.ptr(basis, ct.c_int32), L.ptr(slot, ct.c_int32),
                                                 ptrs, L.ptr(status, ct.c_int32)))
        for i, it in enumerate(items):
            if status[i] == 0:
                self._n_modes[(int(basis[i]), int(slot[i]))] = int(descs[i].n_modes)
                self._n_particles[(int(basis[i]), int(slot[i]))] = int(descs[i].n_particles)
        return status

    def clear_instance(self, basis: int, slot: int) -> None:
        L.check(self.lib.psf_batch_clear_instance(self.handle, int(basis), int(slot)))
        self._n_modes.pop((basis, slot), None)
        self._n_particles.pop((basis, slot), None)

    # ------------------------------------------------------------ stepping
    def step(self, n: int = 1) -> None:
        L.check(self.lib.psf_batch_step(self.handle, int(n)))

    def sync(self) -> None:
        L.check(self.lib.psf_batch_sync(self.handle))

    @property
    def stream(self) -> int:
        s = ct.c_void_p()
        L.check(self.lib.psf_batch_get_stream(self.handle, ct.byref(s)))
        return int(s.value or 0)

    def profile_step(self) -> np.ndarray:
        """Device ms of each launch of one step: [tensor-core step, tracer] when fused."""
        n = self.info()["kernels_per_step"]
        out = np.zeros(n, dtype=np.float64)
        L.check(self.lib.psf_batch_profile_step(self.handle, out.ctypes.data_as(ct.POINTER(ct.c_double)), n))
        return out

    def profile_phases(self) -> np.ndarray:
        """Device ms of [contraction, state update, reconstruction, tracer] run as separate launches."""
        out = np.zeros(4, dtype=np.float64)
        L.check(self.lib.psf_batch_profile_phases(self.handle, out.ctypes.data_as(ct.POINTER(ct.c_double)), 4))
        return out

    def info(self) -> dict:
        i = LB.BatchInfo()
        L.check(self.lib.psf_batch_info_get(self.handle, ct.byref(i)))
        return {k: getattr(i, k) for k, _ in LB.BatchInfo._fields_}

    def pool_free(self) -> tuple[int, int]:
        """(free particles in the pool, largest contiguous free range)."""
        f, l = ct.c_int64(), ct.c_int64()
        L.check(self.lib.psf_batch_pool_free(self.handle, ct.byref(f), ct.byref(l)))
        return int(f.value), int(l.value)

    def device_status(self) -> int:
        c = ct.c_int32()
        L.check(self.lib.psf_batch_device_status(self.handle, ct.byref(c)))
        return int(c.value)

    # ------------------------------------------------------------- results
    def get_state(self, basis: int, slot: int, out=None) -> np.ndarray:
        n = self._n_modes.get((basis, slot), self.bases[basis].n_modes)
        out = np.empty(n, dtype=np.float64) if out is None else out
        L.check(self.lib.psf_batch_get_state(self.handle, int(basis), int(slot), out.ctypes.data, n))
        return out

    def get_particles(self, basis: int, slot: int, out=None) -> np.ndarray:
        P = self._n_particles.get((basis, slot), 0)
        out = np.empty((P, 4), dtype=np.float32) if out is None else out
        L.check(self.lib.psf_batch_get_particles(self.handle, int(basis), int(slot), out.ctypes.data, P))
        return out

    def get_velocity(self, basis: int, slot: int) -> np.ndarray:
        nf = self.bases[basis].n_faces
        out = np.empty(nf, dtype=np.float32)
        L.check(self.lib.psf_batch_get_velocity(self.handle, int(basis), int(slot), out.ctypes.data, nf))
        return out

    def get_steps(self, basis: int, slot: int) -> int:
        s = ct.c_int64()
        L.check(self.lib.psf_batch_get_steps(self.handle, int(basis), int(slot), ct.byref(s)))
        return int(s.value)
