"""Per-domain precompute: eigenbasis and advection tensor (psfsolver.cpp:236-551)."""
import numpy as np
import pytest

from oracle.dec_literal import LiteralDEC, literal_advection
from parallelspectralfluids3d_b200 import basis as B
from parallelspectralfluids3d_b200.domain import box_domain, sphere_obstacle_domain
from parallelspectralfluids3d_b200.fixture import Basis, build_basis

DOMS = [box_domain(6), sphere_obstacle_domain(10, 2.5), sphere_obstacle_domain((12, 10, 9), 3.0),
        box_domain((5, 7, 6))]


@pytest.mark.parametrize("dom", DOMS, ids=lambda d: d.name)
def test_null_space_generators_span_the_null_space(dom):
    K = B.laplacian_interior(dom).toarray()
    w = np.linalg.eigvalsh(K)
    Z, _ = B.null_space_generators(dom)
    Z = Z.toarray()
    assert np.abs(K @ Z).max() < 1e-10
    assert np.linalg.matrix_rank(Z) == int((w <= 1e-10).sum())


@pytest.mark.parametrize("dom", DOMS, ids=lambda d: d.name)
def test_eigenbasis_matches_dense_solver(dom):
    K = B.laplacian_interior(dom).toarray()
    w = np.linalg.eigvalsh(K)
    nz = w[w > 1e-10]
    lam, phi = B.eigenbasis(dom, 10)
    assert np.allclose(lam, nz[:10], rtol=0, atol=1e-10)
    assert np.allclose(phi.T @ phi, np.eye(10), atol=1e-8)
    assert np.allclose(K @ phi, phi * lam, atol=1e-8)


@pytest.mark.parametrize("dom", [box_domain(4), sphere_obstacle_domain((6, 5, 4), 1.2)], ids=lambda d: d.name)
def test_tensor_builder_matches_literal_loop(dom):
    dom.build()
    N = 6
    lam, phi_I = B.eigenbasis(dom, N)
    phi = np.zeros((dom.n_faces, N))
    phi[dom.interior_faces] = phi_I
    psi = B.curl_basis(dom, phi)
    C = B.advection_tensor(dom, phi, psi, lam)
    C_lit = literal_advection(LiteralDEC(dom.dims), dom.inside, dom.h, phi, psi, lam)
    assert np.abs(C - C_lit).max() <= 1e-12 * np.abs(C_lit).max()


def test_tensor_structure_and_prefix_slice(small_bases):
    b = small_bases["sphere12x10x9"]
    A = b.lam[:, None, None] * b.C
    # The wedge bracket is antisymmetric in (k, j).
    assert np.abs(A + A.transpose(2, 1, 0)).max() <= 1e-12 * np.abs(A).max()
    # A prefix of the basis gives the prefix of the tensor.
    dom = b.domain().build()
    n = 9
    phi = b.phi_full()[:, :n]
    C = B.advection_tensor(dom, phi, B.curl_basis(dom, phi), b.lam[:n])
    assert np.abs(C - b.C[:n, :n, :n]).max() <= 1e-13 * np.abs(C).max()
    t = b.truncate(n)
    assert t.n_modes == n and np.array_equal(t.C, b.C[:n, :n, :n])


def test_basis_file_round_trip(tmp_path, small_bases):
    b = small_bases["box576"]
    p = str(tmp_path / "b.psfb")
    b.save(p)
    c = Basis.load(p)
    assert c.dims == b.dims and c.h == b.h
    for f in ("active_faces", "lam", "gravity", "phi", "C", "sign_bits", "inside", "aabb_min", "aabb_max"):
        assert np.array_equal(getattr(b, f), getattr(c, f)), f


def test_gravity_projection(small_bases):
    b = small_bases["box6"]
    dom = b.domain().build()
    phi = b.phi_full()
    g = np.zeros(dom.n_faces)
    ny_ = dom.face_normal[:, 1]
    m = dom.face_inside & (ny_ != 0)
    g[m] = np.where(ny_[m] > 0, 1.0, -1.0) * 0.00981
    assert np.allclose(b.gravity, phi.T @ g)


def test_compact_basis_file_round_trip(tmp_path, small_bases):
    """A .psfc keeps Phi as FP32 and rebuilds C from it on load."""
    from parallelspectralfluids3d_b200.fixture import Basis

    b = small_bases["sphere12x10x9"]
    path = str(tmp_path / "b.psfc")
    b.save(path, compact=True)
    c = Basis.load(path, device="cpu")
    assert np.array_equal(c.phi, b.phi.astype(np.float32).astype(np.float64))
    assert np.array_equal(c.lam, b.lam) and np.array_equal(c.active_faces, b.active_faces)
    assert np.abs(c.C - b.C).max() <= 1e-5 * np.abs(b.C).max()
    # C of the loaded basis is the tensor of its own Phi: rebuilding again gives the same array.
    from parallelspectralfluids3d_b200.fixture import rebuild_tensor

    assert np.array_equal(rebuild_tensor(c, "cpu"), c.C)
