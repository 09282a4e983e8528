"""Per-domain precompute: Laplacian eigenbasis and advection structure tensor.

This produces the inputs of the per-step hot path (Phi, lambda, C, gravity).
It restates the reference's ``buildLaplace`` / ``buildAdvection``
(Solver/SolverImpl/psfsolver.cpp:236-551):

* ``mat = d1^T *1dual d1 *2`` (psfsolver.cpp:247) with the rows of faces that
  do not have exactly two INSIDE voxels removed (psfsolver.cpp:251-265).  The
  primal star on faces is the constant ``1/(2h)`` (DEC/dec.cpp:139-193), so the
  pruned operator restricted to the interior faces I is the symmetric PSD
  matrix ``K = (1/2h) d1_I^T *1dual d1_I``; its eigenpairs with non-zero
  eigenvalue are exactly those of the pruned matrix, padded with zeros.
* The reference takes the lowest ``N`` eigenpairs with eigenvalue > 1e-10
  from a shift-invert Arnoldi solver (Spectra ``GenEigsRealShiftSolver``,
  psfsolver.cpp:273-341).  Spectra and Eigen are not available here; SciPy's
  ARPACK ``eigsh`` in shift-invert mode stands in.  Because the pruned rows
  keep the circulation around wall edges, ``K``'s null space is not all
  gradients (see :func:`null_space_generators`); it is moved above the wanted
  band by adding ``alpha * Z Z^T``, which vanishes on every eigenvector of
  ``K`` with a non-zero eigenvalue, so the returned pairs are eigenpairs of
  ``K`` itself (checked).
* ``Psi = curl Phi`` with ``curl = d1 *2`` (psfsolver.cpp:252, 342).
* gravity on INSIDE y-faces, projected ``g <- Phi^T g`` (psfsolver.cpp:344-358).
* the advection tensor (psfsolver.cpp:431-551)::

      C[k][a][j] = (1/lambda_k) sum_e Psi[e,a] W_k[e,j]
      W_k[e,j]   = sum_{terms t on edge e} s_t (Phi_k[fa_t] Phi_j[fb_t] - Phi_j[fa_t] Phi_k[fb_t])

  with the 12 wedge terms per INSIDE voxel, ``s_t = (h/2)^2 (n_fa x n_fb).(1,1,1)``
  using the faces' stored normals and the edges of the faces' stored ``e1..e4``
  lists.  The reference materialises ``W_k`` densely (O(N^2 E) doubles);
  here the 12 V terms are gathered once and ``C`` is formed with
  ``N`` GEMMs of shape ``N x T x N`` (torch, FP64, on any device), using the
  antisymmetry of the bracket in (k, j) to compute one product only.

Truncating a basis to ``N' < N`` modes is an exact prefix slice of Phi,
lambda, g and C (C[k][a][j] depends only on modes k, a, j).
"""

from __future__ import annotations

import numpy as np

from .domain import Domain

# Per-voxel wedge terms (edge slot, face a, face b), psfsolver.cpp:520-533.
# Edge slots: 0-3 = f1.e1..e4, 4-7 = f2.e1..e4, 8 = f5.e1, 9 = f5.e3,
# 10 = f6.e1, 11 = f6.e3 (psfsolver.cpp:456-467).  Faces 0..5 = f1..f6.
WEDGE_TERMS = (
    (0, 0, 3),
    (1, 5, 0),
    (2, 2, 0),
    (3, 0, 4),
    (4, 3, 1),
    (5, 4, 1),
    (6, 1, 2),
    (7, 1, 5),
    (8, 4, 3),
    (9, 2, 4),
    (10, 3, 5),
    (11, 5, 2),
)

# Gravity magnitude of the reference's CPU solver (psfsolver.cpp:353).
GRAVITY_CPU = 0.00981


def laplacian_interior(dom: Domain):
    """``K = (1/2h) d1_I^T *1dual d1_I`` on the interior faces, as a CSR matrix."""
    import scipy.sparse as sp

    dom.build()
    d1 = dom.d1().tocsc()
    I = dom.interior_faces
    d1I = d1[:, I]
    star = sp.diags(dom.dual_hodge_edges())
    K = (d1I.T @ star @ d1I) * dom.primal_hodge_faces()
    return K.tocsr()


def gradient_interior(dom: Domain):
    """``G = d2^T`` restricted to interior faces x INSIDE voxels."""
    dom.build()
    d2 = dom.d2().tocsc()
    vids = np.nonzero(dom.inside.ravel())[0]
    return d2[vids, :][:, dom.interior_faces].T.tocsr()


def null_space_generators(dom: Domain):
    """Potentials whose gradients span the null space of the pruned operator.

    The pruned rows keep the circulation around INSIDE edges that touch a
    non-interior face ("wall edges"), so the operator does not annihilate
    every gradient.  Around a wall edge the fluid voxels form a chain, and the
    circulation of a gradient over the chain's interior faces telescopes to the
    potential difference of the chain's two end voxels.  The null space is
    therefore spanned by the gradients of indicator potentials of the connected
    components of the graph "end voxels of the same wall edge" (voxels in no
    such pair are their own component).

    Returns ``(Z, singleton)``: a sparse (interior faces x components) matrix
    and a mask of the components that hold a single voxel.
    """
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components

    dom.build()
    interior = np.zeros(dom.n_faces, dtype=bool)
    interior[dom.interior_faces] = True
    wall_edge = np.zeros(dom.n_edges, dtype=bool)
    wall_edge[dom.face_edges[~interior].ravel()] = True
    wall_edge &= dom.edge_inside
    vids = np.nonzero(dom.inside.ravel())[0]
    d1 = dom.d1().tocsr()
    d2 = dom.d2().tocsc()
    G = d2[vids, :][:, dom.interior_faces].T.tocsr()  # interior faces x inside voxels
    B = (d1[np.nonzero(wall_edge)[0], :][:, dom.interior_faces] @ G).tocsr()
    B.eliminate_zeros()
    nnz = np.diff(B.indptr)
    if not np.all((nnz == 0) | (nnz == 2)):
        raise RuntimeError("wall-edge circulation does not telescope to two voxels")
    rows = np.nonzero(nnz == 2)[0]
    u = B.indices[B.indptr[rows]]
    w = B.indices[B.indptr[rows] + 1]
    nv = len(vids)
    graph = sp.coo_matrix((np.ones(len(rows)), (u, w)), shape=(nv, nv))
    ncomp, label = connected_components(graph, directed=False)
    ind = sp.csr_matrix((np.ones(nv), (np.arange(nv), label)), shape=(nv, ncomp))
    singleton = np.bincount(label, minlength=ncomp) == 1
    return (G @ ind).tocsr(), singleton


def nested_dissection_order(A, xyz: np.ndarray, leaf: int = 64) -> np.ndarray:
    """Fill-reducing symmetric ordering for a grid operator.

    Geometric nested dissection: split the vertex set at the median of its
    longest coordinate extent, take as separator the right-hand vertices that
    couple to the left half, order ``[left, right, separator]`` recursively.
    """
    A = A.tocsr()
    n = A.shape[0]
    side = np.zeros(n, dtype=np.int8)
    out = []
    work = [("split", np.arange(n))]
    # Explicit stack: ("split", S) expands to children; ("emit", S) appends.
    while work:
        kind, S = work.pop()
        if kind == "emit":
            out.append(S)
            continue
        if len(S) <= leaf:
            out.append(S)
            continue
        c = xyz[S]
        ax = int(np.argmax(c.max(axis=0) - c.min(axis=0)))
        med = np.median(c[:, ax])
        left = c[:, ax] < med
        if left.all() or not left.any():
            out.append(S)
            continue
        side[S[left]] = 1
        R = S[~left]
        sub = A[R]
        touch = np.zeros(len(R), dtype=bool)
        nz_rows = np.repeat(np.arange(len(R)), np.diff(sub.indptr))
        touch[nz_rows[side[sub.indices] == 1]] = True
        side[S[left]] = 0
        # Post-order: left, right interior, then separator.
        work.append(("emit", R[touch]))
        work.append(("split", R[~touch]))
        work.append(("split", S[left]))
    return np.concatenate(out)


def eigenbasis(dom: Domain, n_modes: int, tol: float = 1e-10):
    """Lowest ``n_modes`` eigenpairs with eigenvalue > 1e-10 of the pruned operator.

    Returns ``(lam, phi_I)``: eigenvalues ascending and unit-norm eigenvectors on
    the interior faces (columns), each with its largest-magnitude entry positive.
    The null-space directions generated by single voxels are lifted by the
    sparse term ``alpha * Zs Zs^T``; the few multi-voxel components stay at
    zero and are requested as extra pairs and then discarded by the reference's
    rule ``lambda > 1e-10`` (psfsolver.cpp:289-290).  Every kept pair is
    checked to be an eigenpair of the pruned operator itself.
    """
    import scipy.sparse as sp
    from scipy.sparse.linalg import LinearOperator, eigsh, splu

    K = laplacian_interior(dom)
    n = K.shape[0]
    Z, singleton = null_space_generators(dom)
    Zs = Z[:, np.nonzero(singleton)[0]]
    n_zero = int((~singleton).sum())
    k = n_modes + n_zero
    if k >= n:
        raise ValueError(f"n_modes={n_modes} exceeds the interior faces of the domain")
    # Smallest Dirichlet eigenvalue of the core Laplacian is about 3 (pi / L)^2.
    L = max(dom.dims)
    alpha = 20.0 / (3.0 * (np.pi / L) ** 2)
    A = (K + alpha * (Zs @ Zs.T)).tocsr()
    sigma = -1e-3
    I = dom.interior_faces
    xyz = dom.face_xyz[I].astype(np.float64) + 0.5
    xyz[np.arange(len(I)), dom.face_axis[I]] -= 0.5
    shifted = (A - sigma * sp.identity(n, format="csr")).tocsr()
    perm = nested_dissection_order(shifted, xyz)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(n)
    lu = splu(shifted[perm][:, perm].tocsc(), permc_spec="NATURAL", diag_pivot_thresh=0.0,
              options={"SymmetricMode": True})

    def solve(x):
        return lu.solve(np.ascontiguousarray(x[perm]))[inv]

    need = n_modes + n_zero
    rng = np.random.default_rng(12345)
    lam, vec = eigsh(LinearOperator((n, n), matvec=A.dot, dtype=np.float64), k=min(n - 1, need + 8),
                     sigma=sigma, which="LM", v0=rng.standard_normal(n), tol=tol,
                     OPinv=LinearOperator((n, n), matvec=solve, dtype=np.float64))
    # Lanczos can miss copies of a repeated eigenvalue (cube symmetries).  Look
    # for missed pairs on A + beta V V^T, whose shifted inverse follows exactly
    # from the factorisation because the columns of V are eigenvectors of A.
    beta = 1e3
    for _ in range(16):
        order = np.argsort(lam)
        lam, vec = lam[order], vec[:, order]
        thr = lam[min(need, lam.size) - 1]
        mu = lam - sigma
        corr = 1.0 / mu - 1.0 / (mu + beta)
        V = vec

        def solve_defl(x, V=V, corr=corr):
            return solve(x) - V @ (corr * (V.T @ x))

        def a_defl(x, V=V):
            return A.dot(x) + beta * (V @ (V.T @ x))

        l2, v2 = eigsh(LinearOperator((n, n), matvec=a_defl, dtype=np.float64), k=8, sigma=sigma,
                       which="LM", v0=rng.standard_normal(n), tol=tol,
                       OPinv=LinearOperator((n, n), matvec=solve_defl, dtype=np.float64))
        missed = l2 < thr - 1e-10 * max(1.0, abs(thr))
        if not missed.any():
            break
        v2 = v2[:, missed]
        v2 = v2 - V @ (V.T @ v2)
        v2, _ = np.linalg.qr(v2)
        lam = np.concatenate([lam, l2[missed]])
        vec = np.concatenate([vec, v2], axis=1)
    else:
        raise RuntimeError("deflation did not converge")
    order = np.argsort(lam)
    lam, vec = lam[order], vec[:, order]
    # Reference acceptance rules (psfsolver.cpp:289-290): lambda > 0, 1/lambda finite.
    keep = lam > 1e-10
    lam, vec = lam[keep][:n_modes], vec[:, keep][:, :n_modes]
    if lam.size < n_modes:
        raise RuntimeError("fewer non-zero eigenpairs than requested")
    res = np.linalg.norm(K @ vec - vec * lam[None, :], axis=0)
    lift = np.linalg.norm(Z.T @ vec, axis=0)
    if not (np.all(res < 1e-7 * np.maximum(1.0, lam)) and np.all(lift < 1e-7)):
        raise RuntimeError("eigenpairs of the lifted operator are not eigenpairs of the pruned one")
    idx = np.argmax(np.abs(vec), axis=0)
    sgn = np.sign(vec[idx, np.arange(vec.shape[1])])
    vec = vec * sgn[None, :]
    return lam, vec


def curl_basis(dom: Domain, phi_full: np.ndarray) -> np.ndarray:
    """``Psi = d1 *2 Phi`` (E x N), psfsolver.cpp:252, 342."""
    return (dom.d1() @ phi_full) * dom.primal_hodge_faces()


def gravity_coefficients(dom: Domain, phi_full: np.ndarray, magnitude: float = GRAVITY_CPU):
    """Gravity on INSIDE y-faces projected on the basis (psfsolver.cpp:344-358)."""
    dom.build()
    g = np.zeros(dom.n_faces)
    ny_ = dom.face_normal[:, 1]
    m = dom.face_inside & (np.abs(ny_) > np.finfo(np.float64).eps)
    g[m] = -np.where(ny_[m] > 0, -1.0, 1.0) * magnitude
    return phi_full.T @ g


def wedge_terms(dom: Domain):
    """Gather the 12 wedge terms of every INSIDE voxel: (edge, face a, face b, weight)."""
    dom.build()
    vids = np.nonzero(dom.inside.ravel())[0]
    vf = dom.voxel_faces[vids]  # (V_in, 6)
    fe = dom.face_edges
    slots = np.concatenate(
        [fe[vf[:, 0]], fe[vf[:, 1]], fe[vf[:, 4]][:, [0, 2]], fe[vf[:, 5]][:, [0, 2]]], axis=1
    )  # (V_in, 12)
    scale = (0.5 * dom.h) ** 2
    edges, fa, fb, wt = [], [], [], []
    ones = np.ones(3)
    for slot, a, b in WEDGE_TERMS:
        na = dom.face_normal[vf[:, a]]
        nb = dom.face_normal[vf[:, b]]
        s = scale * (np.cross(na, nb) @ ones)
        edges.append(slots[:, slot])
        fa.append(vf[:, a])
        fb.append(vf[:, b])
        wt.append(s)
    return (
        np.concatenate(edges),
        np.concatenate(fa),
        np.concatenate(fb),
        np.concatenate(wt),
    )


def advection_tensor(dom: Domain, phi_full: np.ndarray, psi: np.ndarray, lam: np.ndarray,
                     device: str = "cpu", k_chunk: int = 8) -> np.ndarray:
    """C[k][a][j] from the gathered wedge terms (FP64)."""
    import torch

    edges, fa, fb, wt = wedge_terms(dom)
    interior = np.zeros(dom.n_faces, dtype=bool)
    interior[dom.interior_faces] = True
    keep = interior[fa] & interior[fb] & (wt != 0.0)
    edges, fa, fb, wt = edges[keep], fa[keep], fb[keep], wt[keep]
    N = phi_full.shape[1]
    dev = torch.device(device)
    A = torch.from_numpy(psi[edges] * wt[:, None]).to(dev)
    P = torch.from_numpy(phi_full[fa]).to(dev)
    Q = torch.from_numpy(phi_full[fb]).to(dev)
    M1 = torch.empty((N, N, N), dtype=torch.float64, device=dev)
    for k0 in range(0, N, k_chunk):
        k1 = min(N, k0 + k_chunk)
        for k in range(k0, k1):
            M1[k] = (A * P[:, k : k + 1]).T @ Q
    # sum_t A[t,a] (P[t,k] Q[t,j] - Q[t,k] P[t,j]) = M1[k,a,j] - M1[j,a,k]
    C = M1 - M1.permute(2, 1, 0)
    C = C / torch.from_numpy(lam).to(dev)[:, None, None]
    return C.cpu().numpy()
