"""GPU precompute (include/psf_precompute.h, parallelspectralfluids3d_b200/precompute.py).

* ``psf_pre_csr_cheb`` against the same product in SciPy (FP64, 1e-13);
* the Chebyshev-filtered eigen-solve against SciPy's shift-invert ARPACK
  (the stand-in for the reference's Spectra solver, psfsolver.cpp:273-341):
  eigenvalues to 1e-10 relative, every degenerate eigenspace spanned to 1e-7
  (the last cluster may be cut by N, as in the reference);
* the advection tensor against the host builder, which is itself checked
  against the reference's literal wedge loop (psfsolver.cpp:445-550) in
  tests/test_basis.py: max difference <= 1e-12 of max |C|;
* a basis built entirely on the GPU stepped through the plain path against
  the FP64 oracle on the same basis.
"""
import numpy as np
import pytest

from parallelspectralfluids3d_b200 import basis as B
from parallelspectralfluids3d_b200 import precompute as P
from parallelspectralfluids3d_b200.domain import box_domain, sphere_obstacle_domain

from test_precompute import assert_same_eigenbasis

pytestmark = pytest.mark.gpu

EIG_TOL = 1e-10     # relative eigenvalue error vs ARPACK
TENSOR_TOL = 1e-12  # max |C_gpu - C_host| / max |C_host|


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("m", [1, 2, 7, 64, 97])
def test_csr_cheb_matches_scipy(m):
    import torch

    dom = sphere_obstacle_domain(10, 2.5)
    K = B.laplacian_interior(dom)
    n = K.shape[0]
    ld = m + (m & 1) + 2
    rng = np.random.default_rng(m)
    Y, X = rng.standard_normal((n, ld)), rng.standard_normal((n, ld))
    A = P.DeviceCSR(K, "cuda")
    out = torch.full((n, ld), 7.0, dtype=torch.float64, device="cuda")
    P.csr_apply(A, _t(Y), out, m=m, alpha=0.7, beta=-1.3, gamma=0.25, X=_t(X))
    want = 0.7 * (K @ Y) - 1.3 * Y + 0.25 * X
    mm = m + (m & 1)
    got = out.cpu().numpy()
    assert np.abs(got[:, :mm] - want[:, :mm]).max() <= 1e-13 * np.abs(want).max()
    assert np.all(got[:, mm:] == 7.0)  # columns beyond the block untouched


def test_csr_rectangular_product():
    """Psi = (1/2h) d1_I Phi: the non-square use (beta = gamma = 0)."""
    import torch

    dom = box_domain(7)
    dom.build()
    D = dom.d1().tocsr()[:, dom.interior_faces] * dom.primal_hodge_faces()
    rng = np.random.default_rng(3)
    Y = rng.standard_normal((D.shape[1], 128))
    out = torch.empty((D.shape[0], 128), dtype=torch.float64, device="cuda")
    P.csr_apply(P.DeviceCSR(D, "cuda"), _t(Y), out, m=128)
    want = D @ Y
    assert np.abs(out.cpu().numpy() - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("make,n", [
    (lambda: box_domain(8), 24),
    (lambda: sphere_obstacle_domain(10, 2.5), 30),
    (lambda: sphere_obstacle_domain((12, 10, 9), 3.0), 37),
    (lambda: box_domain(12), 160),
])
def test_gpu_eigenbasis_matches_arpack(make, n):
    dom = make()
    lam, phi, stats = P.eigenbasis(dom, n, device=0)
    lam_ref, phi_ref = B.eigenbasis(dom, n)
    assert_same_eigenbasis(lam, phi, lam_ref, phi_ref, tol_lam=EIG_TOL)
    assert stats["max_rel_residual"] < 1e-9 and stats["orthonormality_error"] < 1e-11


@pytest.mark.parametrize("name", ["box16_n64", "sphere12x10x9_n37"])
def test_gpu_tensor_matches_host_builder(name, c1_basis, small_bases):
    b = c1_basis if name == "box16_n64" else small_bases["sphere12x10x9"]
    dom = b.domain()
    dom.build()
    got = P.advection_tensor(dom, b.phi, b.lam, device=0)
    phi_full = b.phi_full()
    want = B.advection_tensor(dom, phi_full, B.curl_basis(dom, phi_full), b.lam)  # host builder, FP64 on the CPU
    assert np.abs(got - want).max() <= TENSOR_TOL * np.abs(want).max()


def test_gpu_tensor_batches_and_splits():
    """Mode batches shorter than N (the last one shorter still) and other edge splits."""
    dom = sphere_obstacle_domain(9, 2.0)
    dom.build()
    lam, phi = B.eigenbasis(dom, 70)
    one = P.advection_tensor(dom, phi, lam, device=0)
    rows = (len(P.wedge_data(dom)[0]) + 15) // 16 * 16
    several = P.advection_tensor(dom, phi, lam, device=0, budget_bytes=rows * 128 * 8 * 9)  # 9 modes per batch
    assert np.abs(one - several).max() <= 1e-13 * np.abs(one).max()  # other edge splits: other rounding
    assert np.array_equal(one, P.advection_tensor(dom, phi, lam, device=0))  # deterministic
    phi_full = np.zeros((dom.n_faces, 70))
    phi_full[dom.interior_faces] = phi
    want = B.advection_tensor(dom, phi_full, B.curl_basis(dom, phi_full), lam)
    assert np.abs(one - want).max() <= TENSOR_TOL * np.abs(want).max()


def test_gpu_built_basis_steps_like_the_oracle():
    """A basis made entirely by the GPU precompute, stepped by the plain path vs the FP64 oracle."""
    from oracle import oracle as O
    from parallelspectralfluids3d_b200 import _lib as L
    from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles
    from parallelspectralfluids3d_b200.solver import Context

    b, stats = P.build_basis(sphere_obstacle_domain(14, 3.5), 96, device=0)
    assert stats["max_rel_residual"] < 1e-9
    w0 = initial_coefficients(b.n_modes, 5)
    parts = initial_particles(b, 4096, 6)
    params = L.make_params(dt=0.01, integrator=L.PSF_RK4)
    with Context(b, params, device=0) as ctx:
        ctx.set_state(w0)
        ctx.set_particles(parts)
        ctx.step(100)
        w = ctx.get_state()
        p = ctx.get_particles()
    ref = O.OracleRollout(b, w0, parts, dt=0.01, integrator=4).step(100)
    assert np.linalg.norm(w - ref.w) / np.linalg.norm(ref.w) <= 1e-5
    assert np.abs(p[:, :3] - ref.pos).max() / b.h <= 1e-3
