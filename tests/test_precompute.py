"""Host logic of the GPU precompute (parallelspectralfluids3d_b200/precompute.py) on the CPU.

The device kernel ``psf_pre_csr_cheb`` is replaced by the same product in
SciPy, so the Chebyshev-filtered subspace iteration (filter, locking,
deflation, Rayleigh-Ritz) is checked here against the shift-invert ARPACK
eigen-solve of :mod:`parallelspectralfluids3d_b200.basis`; the per-edge wedge
data is checked by contracting it in NumPy exactly as the tensor kernels do
and comparing with the host tensor builder (the restatement of
Solver/SolverImpl/psfsolver.cpp:431-551).  The kernels themselves are tested
on the GPU in tests/test_gpu_precompute.py.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from parallelspectralfluids3d_b200 import basis as B
from parallelspectralfluids3d_b200 import precompute as P
from parallelspectralfluids3d_b200.domain import box_domain, sphere_obstacle_domain


@pytest.fixture
def cpu_kernel(monkeypatch):
    """psf_pre_csr_cheb restated with SciPy on CPU tensors."""
    import torch

    class HostCSR:
        def __init__(self, A, device):
            self.A = sp.csr_matrix(A)
            self.n_rows, self.n_cols = A.shape

    def apply(A, Y, out, m=None, alpha=1.0, beta=0.0, gamma=0.0, X=None):
        m = Y.shape[1] if m is None else m
        m2 = m + (m & 1)
        y = Y[:, :m2].numpy()
        r = alpha * (A.A @ y)
        if beta:
            r = r + beta * y
        if gamma:
            r = r + gamma * X[:, :m2].numpy()
        out[:, :m2] = torch.from_numpy(np.ascontiguousarray(r))
        return out

    monkeypatch.setattr(P, "DeviceCSR", HostCSR)
    monkeypatch.setattr(P, "csr_apply", apply)


def clusters(lam, rel=1e-8):
    """Index ranges of (numerically) equal eigenvalues."""
    out, s = [], 0
    for i in range(1, len(lam) + 1):
        if i == len(lam) or lam[i] - lam[i - 1] > rel * lam[i]:
            out.append((s, i))
            s = i
    return out


def assert_same_eigenbasis(lam, vec, lam_ref, vec_ref, tol_lam=1e-10, tol_vec=1e-7):
    """Eigenvalues equal; the spans of every degenerate cluster equal (the last cluster may be cut)."""
    np.testing.assert_allclose(lam, lam_ref, rtol=tol_lam)
    for s, e in clusters(lam_ref)[:-1]:
        P1 = vec[:, s:e] @ vec[:, s:e].T
        P2 = vec_ref[:, s:e] @ vec_ref[:, s:e].T
        assert np.abs(P1 - P2).max() < tol_vec, f"cluster {s}:{e}"


@pytest.mark.parametrize("make,n", [(lambda: box_domain(8), 24), (lambda: sphere_obstacle_domain(10, 2.5), 30)])
def test_chfsi_matches_shift_invert_arpack(cpu_kernel, make, n):
    dom = make()
    K = B.laplacian_interior(dom)
    lam, vec, stats = P.chfsi(K, n, device="cpu", degree=40)
    lam_ref, vec_ref = B.eigenbasis(dom, n)
    assert_same_eigenbasis(lam, vec.numpy(), lam_ref, vec_ref)
    assert stats["outer"] < 100


def test_chfsi_excludes_the_null_space(cpu_kernel):
    """K has a large null space below the wanted band (the gradients of the
    potentials of basis.null_space_generators); none of it is returned."""
    dom = sphere_obstacle_domain(8, 2.0)
    K = B.laplacian_interior(dom)
    lam, vec, _ = P.chfsi(K, 12, device="cpu", degree=30)
    v = vec.numpy()
    assert lam.min() > 1e-3
    Z, _ = B.null_space_generators(dom)
    assert Z.shape[1] > 100
    Zn = Z.multiply(1.0 / np.sqrt(np.asarray(Z.multiply(Z).sum(axis=0)))).tocsr()
    assert np.abs(Zn.T @ v).max() < 1e-9


@pytest.mark.parametrize("make,n", [(lambda: box_domain(6), 12), (lambda: sphere_obstacle_domain((9, 8, 7), 2.0), 15)])
def test_wedge_data_contracts_to_the_host_tensor(make, n):
    dom = make()
    dom.build()
    lam, phi_I = B.eigenbasis(dom, n)
    phi_full = np.zeros((dom.n_faces, n))
    phi_full[dom.interior_faces] = phi_I
    want = B.advection_tensor(dom, phi_full, B.curl_basis(dom, phi_full), lam)
    uniq, faces, S = P.wedge_data(dom)
    rows = np.vstack([phi_I, np.zeros((1, n))])
    psi = (dom.d1().tocsr()[uniq][:, dom.interior_faces] @ phi_I) * dom.primal_hodge_faces()
    F = rows[faces]                                         # (E, 8, N)
    q = np.einsum("efg,efk->egk", S, F)                     # q_e[g][k]
    W = np.einsum("egk,egj->ekj", q, F)                     # W_k[e][j]
    got = np.einsum("ea,ekj->kaj", psi, W) / lam[:, None, None]
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_wedge_data_is_antisymmetric_and_fits_the_slots():
    dom = sphere_obstacle_domain(9, 2.0)
    dom.build()
    uniq, faces, S = P.wedge_data(dom)
    assert np.allclose(S, -np.transpose(S, (0, 2, 1)))
    assert faces.shape[1] == P.WEDGE_SLOTS and faces.max() <= len(dom.interior_faces)
    used = (faces < len(dom.interior_faces)).sum(axis=1)
    assert used.max() == 5  # one term in twelve names a face off its edge
