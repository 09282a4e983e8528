"""Python host mirror of the reference's solver plug-in interface.

``Context`` is a thin owner of one ``psf_ctx`` (include/psf_b200.h).
``PSFSolverCUDA`` mirrors ``AbstractSolver`` (Solver/abstractsolver.h:13-127):
same method names, argument meaning and call order, so code written against
the reference's ``PSFSolver`` / ``PSFSolverGPU`` reads the same.  The mesh
voxelisation and the eigen/tensor precompute run once per domain
(:mod:`parallelspectralfluids3d_b200.fixture`), the way ``setMesh`` /
``buildLaplace`` / ``buildAdvection`` do in the reference
(Solver/abstractsolver.cpp:92-166).
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib as L


class Context:
    """One device context of the single-instance engine."""

    def __init__(self, basis, params: L.Params | None = None, device: int = 0, forcing=None):
        self.lib = L.load()
        self.basis = basis
        self._arrays = L.BasisArrays(basis)
        self.params = params or L.make_params()
        self.handle = ct.c_void_p()
        L.check(self.lib.psf_create(ct.byref(self._arrays.desc), ct.byref(self.params), int(device),
                                    ct.byref(self.handle)))
        self.N = basis.n_modes
        self.n_faces = basis.n_faces
        self.P = 0
        if forcing is not None:
            self.set_forcing(forcing)

    def close(self) -> None:
        if self.handle:
            L.check(self.lib.psf_destroy(self.handle))
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

    # ------------------------------------------------------------- state
    def set_params(self, params: L.Params) -> None:
        L.check(self.lib.psf_set_params(self.handle, ct.byref(params)))
        self.params = params

    def set_state(self, w) -> None:
        w = np.ascontiguousarray(w, dtype=np.float64)
        L.check(self.lib.psf_set_state(self.handle, w.ctypes.data, int(w.shape[0])))

    def get_state(self, out=None) -> np.ndarray:
        out = np.empty(self.N, dtype=np.float64) if out is None else out
        L.check(self.lib.psf_get_state(self.handle, out.ctypes.data, int(self.N)))
        return out

    def set_forcing(self, f) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64)
        L.check(self.lib.psf_set_forcing(self.handle, f.ctypes.data, int(f.shape[0])))

    def set_particles(self, parts) -> None:
        parts = np.ascontiguousarray(parts, dtype=np.float32).reshape(-1, 4)
        L.check(self.lib.psf_set_particles(self.handle, parts.ctypes.data, int(parts.shape[0])))
        self.P = int(parts.shape[0])

    def get_particles(self, out=None) -> np.ndarray:
        out = np.empty((self.P, 4), dtype=np.float32) if out is None else out
        L.check(self.lib.psf_get_particles(self.handle, out.ctypes.data, int(self.P)))
        return out

    def get_velocity(self) -> np.ndarray:
        out = np.empty(self.n_faces, dtype=np.float32)
        L.check(self.lib.psf_get_velocity(self.handle, out.ctypes.data, int(self.n_faces)))
        return out

    # ------------------------------------------------------------ stepping
    def step(self, n: int = 1) -> None:
        L.check(self.lib.psf_step(self.handle, int(n)))

    def sync(self) -> None:
        L.check(self.lib.psf_sync(self.handle))

    @property
    def stream(self) -> int:
        s = ct.c_void_p()
        L.check(self.lib.psf_get_stream(self.handle, ct.byref(s)))
        return int(s.value or 0)

    def profile_step(self) -> np.ndarray:
        """Run one step kernel by kernel; device milliseconds per kernel."""
        n = self.kernels_per_step()
        out = np.zeros(n, dtype=np.float64)
        L.check(self.lib.psf_profile_step(self.handle, out.ctypes.data_as(ct.POINTER(ct.c_double)), n))
        return out

    def kernels_per_step(self) -> int:
        n = ct.c_int32()
        L.check(self.lib.psf_kernels_per_step(self.handle, ct.byref(n)))
        return int(n.value)


class PSFSolverCUDA:
    """``AbstractSolver`` mirror backed by the CUDA engine.

    Defaults follow the reference constructor (Solver/abstractsolver.cpp:7-46):
    ``N = 16``, ``dt = 1/60``, ``viscosity = 0``, lifetime ``60`` steps,
    gravity off, forward-Euler particles.
    """

    def __init__(self, device: int = 0):
        self.device = device
        self.nEigenFunctions = 16
        self.timeStep = 1.0 / 60.0
        self.viscosity = 0.0
        self.lifeTime = 1.0 * 60.0
        self.gravityActive = False
        self.integrator = L.PSF_RK1
        self.flags = L.PSF_FLAG_RENORM
        self.seed = 0
        self.maxParticles = 1000
        self.full_basis = None
        self.basis = None
        self.ctx: Context | None = None
        self.basisCoeff = None
        self.particles = np.zeros((0, 4), dtype=np.float32)
        self.simTime = 0.0

    # ------------------------------------------------ precompute / layout
    def setMesh(self, basis) -> None:
        """Attach a precomputed domain basis (replaces voxelise + buildLaplace + buildAdvection)."""
        self.full_basis = basis
        self.nEigenFunctions = min(self.nEigenFunctions, basis.n_modes)
        self.buildLaplace()
        self.buildAdvection()

    def buildLaplace(self) -> None:
        self.basis = self.full_basis.truncate(self.nEigenFunctions)
        self.basisCoeff = np.zeros(self.nEigenFunctions)

    def buildAdvection(self) -> None:
        if self.ctx is not None:
            self.ctx.close()
        self.ctx = Context(self.basis, self._params(), device=self.device)
        self.ctx.set_forcing(self.basis.gravity)
        self.ctx.set_state(self.basisCoeff)
        self.ctx.set_particles(self.particles)

    def _params(self) -> L.Params:
        flags = self.flags | (L.PSF_FLAG_FORCING if self.gravityActive else 0)
        return L.make_params(dt=self.timeStep, viscosity=self.viscosity, lifetime=self.lifeTime,
                             integrator=self.integrator, flags=flags, seed=self.seed)

    def _push_params(self) -> None:
        if self.ctx is not None:
            self.ctx.set_params(self._params())

    # ------------------------------------------------------ the plug-in
    def integrate(self) -> None:
        """One step (Solver/SolverImpl/psfsolver.cpp:21-234)."""
        self.ctx.step(1)
        self.simTime += 1.0

    # ------------------------------------------------------------ setters
    def setInitialVelocityField(self, field) -> None:
        """``basisCoeff = Phi^T field`` (Solver/abstractsolver.cpp:168-171)."""
        f = np.asarray(field, dtype=np.float64)
        w = self.basis.phi.T @ f[self.basis.active_faces]
        self.setBasisCoefficients(w)

    def setBasisCoefficients(self, w) -> None:
        self.basisCoeff = np.array(w, dtype=np.float64)
        self.ctx.set_state(self.basisCoeff)

    def setNumberEigenFunctions(self, n: int) -> None:
        self.nEigenFunctions = int(n)
        if self.full_basis is not None:
            self.buildLaplace()
            self.buildAdvection()

    def changeNumParticles(self, n: int) -> None:
        self.maxParticles = int(n)
        self.clearParticles()

    def setViscosity(self, visc: float) -> None:
        self.viscosity = float(visc)
        self._push_params()

    def setTimestep(self, timestep: float) -> None:
        self.timeStep = float(timestep)
        self._push_params()

    def setGravityActive(self, state: bool) -> None:
        self.gravityActive = bool(state)
        self._push_params()

    def setLifeTime(self, lt: float) -> None:
        """Lifetime in seconds at 60 steps per second (Solver/abstractsolver.cpp:238-241)."""
        self.lifeTime = float(lt) * 60.0
        self._push_params()

    def setIntegrator(self, integrator: int) -> None:
        self.integrator = int(integrator)
        self._push_params()

    def setForcing(self, f) -> None:
        self.ctx.set_forcing(f)

    # ------------------------------------------------------------ getters
    def getNumEigenFunctions(self) -> int:
        return self.nEigenFunctions

    def getTimestep(self) -> float:
        return self.timeStep

    def getEigenFunction(self, n: int) -> np.ndarray:
        return self.basis.phi_full()[:, n]

    def getVelocityBasisField(self) -> np.ndarray:
        return self.basis.phi_full()

    def getBasisCoefficients(self) -> np.ndarray:
        return self.ctx.get_state()

    def getVelocityField(self) -> np.ndarray:
        return self.ctx.get_velocity()

    def getParticles(self) -> np.ndarray:
        return self.ctx.get_particles()

    def getNumParticles(self) -> int:
        return self.ctx.P if self.ctx else 0

    def setParticles(self, parts) -> None:
        self.particles = np.ascontiguousarray(parts, dtype=np.float32).reshape(-1, 4)
        if self.ctx is not None:
            self.ctx.set_particles(self.particles)

    def clearParticles(self) -> None:
        self.simTime = 0.0
        self.particles = np.zeros((0, 4), dtype=np.float32)
        if self.ctx is not None:
            self.ctx.set_particles(self.particles)
