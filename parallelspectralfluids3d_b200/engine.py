"""Python host side of the serving engine (``include/psf_engine.h``).

:class:`Engine` accepts rollout requests from any thread; its native worker
admits them into free batch slots as slots, particle-pool ranges and the
device-memory budget allow, steps all admitted rollouts together, and
retires each one at its own step count (continuous batching).
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib as L
from . import _lib_engine as LE


class Engine:
    def __init__(self, bases, slots, max_particles: int, particle_pool: int = 0, hbm_budget_bytes: int = 0,
                 chunk_steps: int = 8, device: int = 0, autotune: bool = True):
        self.lib = L.load()
        n = len(bases)
        slots = [int(slots)] * n if np.isscalar(slots) else [int(s) for s in slots]
        self.bases = list(bases)
        self._arrays = [L.BasisArrays(b) for b in bases]
        descs = (L.BasisDesc * n)(*[a.desc for a in self._arrays])
        self._slots = (ct.c_int32 * n)(*slots)
        cfg = LE.EngineConfig()
        cfg.n_bases = n
        cfg.bases = descs
        cfg.slots = self._slots
        cfg.max_particles = int(max_particles)
        cfg.particle_pool = int(particle_pool)
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.chunk_steps = int(chunk_steps)
        cfg.autotune = 1 if autotune else 0
        self.handle = ct.c_void_p()
        L.check(self.lib.psf_engine_create(ct.byref(cfg), int(device), ct.byref(self.handle)))
        self._meta = {}

    def close(self) -> None:
        if self.handle:
            L.check(self.lib.psf_engine_destroy(self.handle))
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

    def submit(self, basis: int, w0, steps: int, params: L.Params, particles=None, forcing=None) -> int:
        w0 = np.ascontiguousarray(w0, dtype=np.float64)
        q = LE.Request()
        q.basis = int(basis)
        q.n_modes = int(w0.shape[0])
        q.steps = int(steps)
        q.params = params
        q.w0 = L.ptr(w0, ct.c_double)
        keep = [w0]
        if forcing is not None:
            f = np.ascontiguousarray(forcing, dtype=np.float64)
            keep.append(f)
            q.forcing = L.ptr(f, ct.c_double)
        P = 0
        if particles is not None:
            p = np.ascontiguousarray(particles, dtype=np.float32).reshape(-1, 4)
            keep.append(p)
            P = int(p.shape[0])
            if P:
                q.particles = L.ptr(p, ct.c_float)
        q.n_particles = P
        rid = ct.c_uint64()
        L.check(self.lib.psf_engine_submit(self.handle, ct.byref(q), ct.byref(rid)))
        self._meta[int(rid.value)] = (int(w0.shape[0]), P)
        return int(rid.value)

    def poll(self, max_ids: int = 1024) -> list[int]:
        ids = (ct.c_uint64 * max_ids)()
        n = ct.c_int32()
        L.check(self.lib.psf_engine_poll(self.handle, ids, int(max_ids), ct.byref(n)))
        return [int(ids[i]) for i in range(n.value)]

    def wait(self, rid: int, timeout_s: float = 60.0) -> bool:
        rc = self.lib.psf_engine_wait(self.handle, int(rid), float(timeout_s))
        if rc == -7:
            return False
        L.check(rc)
        return True

    def collect(self, rid: int, want_particles: bool = True):
        """(w, particles or None, info dict) of a finished request."""
        n, P = self._meta.pop(rid)
        w = np.empty(n, dtype=np.float64)
        p = np.empty((P, 4), dtype=np.float32) if want_particles else None
        info = LE.RequestInfo()
        L.check(self.lib.psf_engine_collect(self.handle, int(rid), w.ctypes.data, n,
                                            p.ctypes.data if p is not None else None, P if p is not None else 0,
                                            ct.byref(info)))
        return w, p, {k: getattr(info, k) for k, _ in LE.RequestInfo._fields_}

    def drain(self, timeout_s: float = 600.0) -> None:
        L.check(self.lib.psf_engine_drain(self.handle, float(timeout_s)))

    def stats(self) -> dict:
        s = LE.EngineStats()
        L.check(self.lib.psf_engine_stats_get(self.handle, ct.byref(s)))
        return {k: getattr(s, k) for k, _ in LE.EngineStats._fields_}
