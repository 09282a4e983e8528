"""The AbstractSolver plug-in on the GPU: the C++ PSFSolverCUDA (headless driver)
and the Python mirror, both against the FP64 oracle."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles
from parallelspectralfluids3d_b200.solver import PSFSolverCUDA

from conftest import ROOT, rel_err

pytestmark = pytest.mark.gpu
TOOL = os.path.join(ROOT, "parallelspectralfluids3d_b200", "psf_run")


@pytest.mark.parametrize("integrator", [1, 4])
def test_cpp_psfsolvercuda_matches_oracle(tmp_path, small_bases, integrator):
    b = small_bases["sphere12x10x9"]
    path = str(tmp_path / "b.psfb")
    b.save(path)
    n = 20
    w0 = initial_coefficients(n, 4)
    parts = initial_particles(b, 640, 5)
    w0.astype("<f8").tofile(tmp_path / "w0.f64")
    parts.astype("<f4").tofile(tmp_path / "p.f32")
    out = str(tmp_path / "out")
    subprocess.run([TOOL, path, str(n), "30", "0.03", str(integrator), str(tmp_path / "w0.f64"),
                    str(tmp_path / "p.f32"), out], check=True)
    w = np.fromfile(out + ".w.f64", dtype="<f8")
    p = np.fromfile(out + ".p.f32", dtype="<f4").reshape(-1, 4)
    ref = O.OracleRollout(b.truncate(n), w0, parts, dt=0.03, integrator=integrator).step(30)
    assert rel_err(w, ref.w) <= 1e-5
    assert np.abs(p[:, :3] - ref.pos).max() / b.h <= 1e-4


def test_cpp_tool_reports_errors(tmp_path):
    r = subprocess.run([TOOL, str(tmp_path / "missing.psfb"), "4", "1", "0.01", "1", "a", "b", "c"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_python_mirror_of_abstract_solver(c1_basis):
    s = PSFSolverCUDA()
    s.setNumberEigenFunctions(48)
    s.setTimestep(0.01)
    s.setMesh(c1_basis)
    assert s.getNumEigenFunctions() == 48
    s.setIntegrator(L.PSF_RK4)
    rng = np.random.default_rng(3)
    field = rng.standard_normal(c1_basis.n_faces)
    s.setInitialVelocityField(field)
    w0 = s.getBasisCoefficients()
    b48 = c1_basis.truncate(48)
    assert np.allclose(w0, b48.phi.T @ field[b48.active_faces])
    parts = initial_particles(c1_basis, 333, 8)
    s.setParticles(parts)
    for _ in range(20):
        s.integrate()
    ref = O.OracleRollout(b48, w0, parts, dt=0.01, integrator=4).step(20)
    assert rel_err(s.getBasisCoefficients(), ref.w) <= 1e-5
    assert np.abs(s.getParticles()[:, :3] - ref.pos).max() / c1_basis.h <= 1e-4
    u = s.getVelocityField()
    assert np.abs(u - ref.u).max() <= 2e-6 * np.abs(ref.u).max()
    # Gravity on: forcing = projected gravity (psfsolver.cpp:56-59).
    s.setGravityActive(True)
    s.integrate()
    ref.force = np.ascontiguousarray(b48.gravity)
    ref.flags |= O.FLAG_FORCING
    ref.step(1)
    assert rel_err(s.getBasisCoefficients(), ref.w) <= 1e-5
