"""Per-domain precompute on the GPU: Laplacian eigenbasis and advection tensor.

Restates the reference's ``PSFSolver::buildLaplace`` and ``buildAdvection``
(Solver/SolverImpl/psfsolver.cpp:236-342 and :431-551) on one GPU, for the
same inputs the host path of :mod:`.basis` uses:

* **Eigen-solve.**  The reference takes the lowest ``N`` eigenpairs with
  eigenvalue > 1e-10 of the pruned 1-form Laplacian with a shift-invert
  Arnoldi solver (Spectra, psfsolver.cpp:273-341).  Its non-zero eigenpairs
  are those of the symmetric interior operator
  ``K = (1/2h) d1_I^T *1dual d1_I`` (:func:`.basis.laplacian_interior`).
  Here they come from Chebyshev-filtered subspace iteration (Zhou, Saad,
  Tiago and Chelikowsky, J. Comput. Phys. 219 (2006) 172-184; the scaled
  filter of Zhou and Saad, SIAM J. Matrix Anal. Appl. 29 (2007) 954-971)
  with locking of converged Ritz pairs.  Every polynomial degree is one
  launch of the hand-written CSR kernel ``psf_pre_csr_cheb``; Rayleigh-Ritz
  and QR of the block are FP64 library calls (cuBLAS / cuSOLVER through
  torch).  ``K``'s null space lies below the wanted band, where a Chebyshev
  filter amplifies most, so every filter starts from ``K X``: that product
  has no null-space component, and the filter's gain at 0 exceeds its gain at
  the lowest wanted eigenvalue by a few percent per pass only.  The result is
  an eigenbasis of ``K`` (checked: residuals, orthonormality), unique up to
  rotations inside degenerate eigenspaces, as the reference's is.
* **Tensor.**  ``C[k][a][j] = (1/lambda_k) sum_e Psi[e][a] W_k[e][j]``
  (psfsolver.cpp:539-550) with the voxels' 12 wedge terms
  (psfsolver.cpp:456-533) gathered per edge into an antisymmetric matrix over
  the faces they name; ``psf_pre_advection_tensor`` generates ``W_k`` for
  batches of modes and contracts it with ``Psi = (1/2h) d1 Phi``
  (psfsolver.cpp:252, 342) by a split-K FP64 GEMM.

There is no CPU fallback here: every function needs the CUDA library and a
device.  The host restatement in :mod:`.basis` is the test reference.
"""

from __future__ import annotations

import ctypes as ct
import time

import numpy as np

from . import _lib as L
from . import basis as B
from ._lib_pre import WedgeDesc
from .domain import Domain

WEDGE_SLOTS = 8  # PSF_WEDGE_SLOTS of include/psf_precompute.h


# ------------------------------------------------------------ device CSR
class DeviceCSR:
    """A scipy CSR matrix held on the device as int32 row pointers / column indices and FP64 values."""

    def __init__(self, A, device):
        import torch

        A = A.tocsr()
        A.sort_indices()
        if A.nnz >= 2**31 or max(A.shape) >= 2**31:
            raise ValueError("matrix too large for 32-bit CSR indices")
        self.n_rows, self.n_cols = A.shape
        self.row_ptr = torch.from_numpy(A.indptr.astype(np.int32)).to(device)
        self.col_idx = torch.from_numpy(A.indices.astype(np.int32)).to(device)
        self.vals = torch.from_numpy(A.data.astype(np.float64)).to(device)


def _stream_ptr(device):
    import torch

    return ct.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def csr_apply(A: DeviceCSR, Y, out, m=None, alpha=1.0, beta=0.0, gamma=0.0, X=None):
    """``out[:, :m] = alpha A Y + beta Y + gamma X`` through ``psf_pre_csr_cheb`` (row-major FP64 blocks)."""
    lib = L.load()
    ld = Y.shape[1]
    m = ld if m is None else m
    for t in (Y, out) + ((X,) if X is not None else ()):
        if not (t.is_contiguous() and t.shape[1] == ld and t.dtype == Y.dtype):
            raise ValueError("blocks must be contiguous FP64 with equal row stride")
    L.check(lib.psf_pre_csr_cheb(A.n_rows, A.n_cols, int(m), int(ld), A.row_ptr.data_ptr(), A.col_idx.data_ptr(),
                                 A.vals.data_ptr(), Y.data_ptr(), X.data_ptr() if X is not None else None,
                                 out.data_ptr(), float(alpha), float(beta), float(gamma), _stream_ptr(Y.device)))
    return out


def gershgorin_bound(K) -> float:
    """An upper bound of the spectrum of a symmetric matrix (largest absolute row sum)."""
    return float(np.abs(K).sum(axis=1).max())


# ----------------------------------------------------------- eigen-solve
def chfsi(K, n_modes: int, device=0, degree: int = 48, guard: int | None = None, tol: float = 1e-10,
          max_outer: int = 300, seed: int = 12345):
    """Lowest ``n_modes`` eigenpairs with non-zero eigenvalue of the symmetric PSD matrix ``K``.

    Returns ``(lam, vec, stats)``: eigenvalues ascending (numpy), eigenvectors
    as a device tensor ``(n, n_modes)`` with orthonormal columns, and the
    iteration statistics.  A pair is converged when
    ``||K v - theta v|| <= tol * theta``; converged pairs are locked in
    ascending order and leave the active block.
    """
    import torch

    dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
    A = DeviceCSR(K, dev)
    n = A.n_rows
    N = int(n_modes)
    guard = max(32, N // 4) if guard is None else int(guard)
    m = N + guard
    if m >= n:
        raise ValueError(f"n_modes={N} plus guard {guard} exceeds the operator size {n}")
    b = gershgorin_bound(K)
    f64 = torch.float64
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)

    def new_block(cols):
        return torch.empty((n, cols + (cols & 1)), dtype=f64, device=dev)

    def apply(Y, cols):
        out = new_block(cols)
        return csr_apply(A, Y, out, m=cols)

    def random_range(cols):
        R = new_block(cols)
        R.normal_(generator=gen)
        if R.shape[1] > cols:
            R[:, cols:] = 0.0
        return apply(R, cols)[:, :cols]

    locked = torch.empty((n, N), dtype=f64, device=dev)
    lam_locked = []
    n_lock = 0

    def deflate(Y):
        if n_lock:
            Lk = locked[:, :n_lock]
            for _ in range(2):
                Y = Y - Lk @ (Lk.T @ Y)
        return Y

    Xa = torch.linalg.qr(random_range(m)).Q
    stats = dict(n=n, nnz=int(K.nnz), guard=guard, degree=degree, bound=b, outer=0, spmm=0, spmm_columns=0)
    t0 = time.perf_counter()
    for outer in range(max_outer):
        ma = Xa.shape[1]
        Xc = new_block(ma)
        Xc[:, :ma] = Xa
        if Xc.shape[1] > ma:
            Xc[:, ma:] = 0.0
        KX = apply(Xc, ma)[:, :ma]
        stats["spmm"] += 1
        stats["spmm_columns"] += ma
        H = Xa.T @ KX
        H = 0.5 * (H + H.T)
        th, Q = torch.linalg.eigh(H)
        Xa = Xa @ Q
        KX = KX @ Q
        res = torch.linalg.vector_norm(KX - Xa * th, dim=0)
        th_h = th.cpu().numpy()
        res_h = res.cpu().numpy()
        null = th_h < 1e-8 * max(th_h.max(), 1e-300)
        conv = (res_h <= tol * np.abs(th_h)) & ~null
        k = 0
        while k < ma and conv[k] and n_lock + k < N:
            k += 1
        if k:
            locked[:, n_lock:n_lock + k] = Xa[:, :k]
            lam_locked.extend(th_h[:k].tolist())
            n_lock += k
            Xa, KX, th_h, null = Xa[:, k:], KX[:, k:], th_h[k:], null[k:]
        stats["outer"] = outer + 1
        if n_lock >= N:
            break
        ma = Xa.shape[1]
        a = float(th_h.max())
        a0 = float(th_h[~null].min()) if (~null).any() else a / 2
        # The filter starts from K X (no null-space component); null Ritz
        # vectors, if any, are replaced by fresh vectors in the range of K.
        Y0 = new_block(ma)
        Y0[:, :ma] = KX
        if null.any():
            idx = torch.from_numpy(np.nonzero(null)[0]).to(dev)
            Y0[:, idx] = random_range(int(null.sum()))
        Y0[:, :ma] /= torch.linalg.vector_norm(Y0[:, :ma], dim=0)
        if Y0.shape[1] > ma:
            Y0[:, ma:] = 0.0
        e = (b - a) / 2.0
        c = (b + a) / 2.0
        sigma = e / (a0 - c)
        tau = 2.0 / sigma
        Xp = Y0
        Y = new_block(ma)
        csr_apply(A, Xp, Y, m=ma, alpha=sigma / e, beta=-c * sigma / e)
        for _ in range(2, degree + 1):
            sn = 1.0 / (tau - sigma)
            Yn = torch.empty_like(Y)
            csr_apply(A, Y, Yn, m=ma, alpha=2.0 * sn / e, beta=-2.0 * c * sn / e, gamma=-sigma * sn, X=Xp)
            Xp, Y, sigma = Y, Yn, sn
        stats["spmm"] += degree
        stats["spmm_columns"] += degree * ma
        Xa = torch.linalg.qr(deflate(Y[:, :ma])).Q
        Xa = torch.linalg.qr(deflate(Xa)).Q
    else:
        raise RuntimeError(f"eigen-solve did not converge in {max_outer} outer iterations ({n_lock}/{N} locked)")
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
    stats["seconds"] = time.perf_counter() - t0
    lam = np.asarray(lam_locked[:N])
    order = np.argsort(lam, kind="stable")
    lam = lam[order]
    vec = locked[:, torch.from_numpy(order).to(dev)]
    return lam, vec, stats


def eigenbasis(dom: Domain, n_modes: int, device=0, **kw):
    """Eigenbasis of the domain's interior operator on the GPU (same contract as :func:`.basis.eigenbasis`).

    Returns ``(lam, phi_I, stats)`` with ``phi_I`` a numpy array (interior
    faces x modes), each column's largest-magnitude entry positive.  Every pair
    is checked: relative residual and orthonormality.
    """
    import torch

    K = B.laplacian_interior(dom)
    lam, vec, stats = chfsi(K, n_modes, device=device, **kw)
    if not np.all(lam > 1e-10):
        raise RuntimeError("eigen-solve returned a null-space vector")
    A = DeviceCSR(K, vec.device)
    n = A.n_rows
    V = torch.zeros((n, n_modes + (n_modes & 1)), dtype=torch.float64, device=vec.device)
    V[:, :n_modes] = vec
    KV = csr_apply(A, V, torch.empty_like(V), m=n_modes)[:, :n_modes]
    lam_t = torch.from_numpy(lam).to(vec.device)
    rel = (torch.linalg.vector_norm(KV - vec * lam_t, dim=0) / lam_t).max().item()
    orth = (vec.T @ vec - torch.eye(n_modes, dtype=torch.float64, device=vec.device)).abs().max().item()
    stats["max_rel_residual"] = rel
    stats["orthonormality_error"] = orth
    if not (rel < 1e-7 and orth < 1e-9):
        raise RuntimeError(f"eigenpairs failed the check: residual {rel:.2e}, orthonormality {orth:.2e}")
    idx = vec.abs().argmax(dim=0)
    sgn = torch.sign(vec[idx, torch.arange(n_modes, device=vec.device)])
    phi = (vec * sgn).cpu().numpy()
    return lam, phi, stats


# ---------------------------------------------------------------- tensor
def wedge_data(dom: Domain):
    """Per-edge wedge data: edge ids, face rows (interior index, or n_interior for none) and S_e.

    ``W_k[e][j] = sum_{f,g} S_e[f][g] Phi[f_e][k] Phi[g_e][j]`` reproduces
    ``sum_t s_t (Phi_k[fa_t] Phi_j[fb_t] - Phi_j[fa_t] Phi_k[fb_t])`` over the
    edge's wedge terms (psfsolver.cpp:520-533).  An edge takes at most four
    terms, one from each voxel around it, but the reference's edge slots pair
    one term in twelve with a face that does not touch the edge, so an edge
    can name five faces; ``WEDGE_SLOTS`` (eight) covers any four terms.
    """
    edges, fa, fb, wt = B.wedge_terms(dom)
    I = dom.interior_faces
    row = np.full(dom.n_faces, -1, dtype=np.int64)
    row[I] = np.arange(len(I))
    keep = (row[fa] >= 0) & (row[fb] >= 0) & (wt != 0.0)
    e, ra, rb, s = edges[keep], row[fa[keep]], row[fb[keep]], wt[keep]
    uniq, einv = np.unique(e, return_inverse=True)
    T = len(e)
    pairs = np.stack([np.concatenate([einv, einv]), np.concatenate([ra, rb])], axis=1)
    up, pinv = np.unique(pairs, axis=0, return_inverse=True)
    pinv = pinv.ravel()
    first = np.searchsorted(up[:, 0], np.arange(len(uniq)))
    pos = np.arange(len(up)) - first[up[:, 0]]
    if pos.max(initial=0) >= WEDGE_SLOTS:
        raise RuntimeError(f"an edge names more than {WEDGE_SLOTS} faces in its wedge terms")
    faces = np.full((len(uniq), WEDGE_SLOTS), len(I), dtype=np.int32)
    faces[up[:, 0], pos] = up[:, 1]
    pa, pb = pos[pinv[:T]], pos[pinv[T:]]
    S = np.zeros((len(uniq), WEDGE_SLOTS, WEDGE_SLOTS))
    np.add.at(S, (einv, pa, pb), s)
    np.add.at(S, (einv, pb, pa), -s)
    return uniq, faces, S


def advection_tensor(dom: Domain, phi_I: np.ndarray, lam: np.ndarray, device=0, budget_bytes: int = 8 << 30,
                     return_device: bool = False, stats: dict | None = None):
    """``C[k][a][j]`` (FP64, ``(N, N, N)``) on the GPU from the interior-face basis ``phi_I``.

    ``stats``, when given, receives the device time of the tensor kernels
    (``kernel_ms``), the edges with wedge terms, the mode batch and the GEMM's
    FP64 operation count (``gemm_flops`` = 2 N^2 ldn E over all batches).
    """
    import torch

    dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
    lib = L.load()
    n, N = phi_I.shape
    ldn = (N + 127) // 128 * 128
    uniq, faces8, S = wedge_data(dom)
    E = len(uniq)
    phi_d = torch.zeros((n + 1, ldn), dtype=torch.float64, device=dev)
    phi_d[:n, :N] = torch.from_numpy(np.ascontiguousarray(phi_I, dtype=np.float64)).to(dev)
    # Psi = (1/2h) d1 Phi on the edges that carry wedge terms (psfsolver.cpp:252, 342).
    D = dom.d1().tocsr()[uniq][:, dom.interior_faces] * dom.primal_hodge_faces()
    psi = torch.empty((max(E, 1), ldn), dtype=torch.float64, device=dev)
    if E:
        csr_apply(DeviceCSR(D, dev), phi_d, psi[:E], m=ldn)
    faces_d = torch.from_numpy(faces8).to(dev)
    S_d = torch.from_numpy(np.ascontiguousarray(S)).to(dev)
    lam_d = torch.from_numpy(np.ascontiguousarray(lam, dtype=np.float64)).to(dev)
    desc = WedgeDesc(E, N, ldn, faces_d.data_ptr(), S_d.data_ptr(), psi.data_ptr(), phi_d.data_ptr(), n,
                     lam_d.data_ptr())
    rows = (E + 15) // 16 * 16
    kb = int(max(1, min(N, 64, budget_bytes // max(1, rows * ldn * 8))))
    ws_bytes = ct.c_int64()
    L.check(lib.psf_pre_advection_workspace(ct.byref(desc), kb, ct.byref(ws_bytes)))
    ws = torch.empty((ws_bytes.value + 255) // 8, dtype=torch.float64, device=dev)
    C = torch.empty((N, N, N), dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    L.check(lib.psf_pre_advection_tensor(ct.byref(desc), kb, ws.data_ptr(), ws_bytes.value, C.data_ptr(),
                                         _stream_ptr(dev)))
    e1.record(st)
    torch.cuda.synchronize(dev)
    if stats is not None:
        stats.update(kernel_ms=e0.elapsed_time(e1), edges=E, k_batch=kb, ldn=ldn,
                     gemm_flops=2.0 * N * (N * ldn) * ((E + 15) // 16 * 16))
    del ws
    return C if return_device else C.cpu().numpy()


def build_basis(dom: Domain, n_modes: int, device=0, **kw):
    """The whole per-domain precompute on the GPU; returns a :class:`.fixture.Basis` and timings."""
    from .fixture import Basis

    t0 = time.perf_counter()
    dom.build()
    t1 = time.perf_counter()
    lam, phi_I, stats = eigenbasis(dom, n_modes, device=device, **kw)
    t2 = time.perf_counter()
    phi_full = np.zeros((dom.n_faces, n_modes))
    phi_full[dom.interior_faces] = phi_I
    grav = B.gravity_coefficients(dom, phi_full)
    tstats = {}
    C = advection_tensor(dom, phi_I, lam, device=device, stats=tstats)
    t3 = time.perf_counter()
    stats.update(domain_s=t1 - t0, eigensolve_s=t2 - t1, tensor_s=t3 - t2,
                 **{f"tensor_{k}": v for k, v in tstats.items()})
    b = Basis(dom.dims, dom.h, dom.aabb_min, dom.aabb_max, dom.interior_faces.astype(np.int32), lam, grav, phi_I,
              C, dom.sign_bits, dom.inside.ravel().astype(np.uint8), name=dom.name)
    return b, stats


def main(argv=None) -> None:
    """Build one domain's basis on the GPU and print its statistics (optionally save it).

    ``python -m parallelspectralfluids3d_b200.precompute box 24 128``
    ``python -m parallelspectralfluids3d_b200.precompute sphere 40 384 --radius 10 --out b.psfb``
    """
    import argparse
    import json

    from .domain import box_domain, channel_domain, sphere_obstacle_domain

    ap = argparse.ArgumentParser(description=main.__doc__.splitlines()[0])
    ap.add_argument("kind", choices=["box", "sphere", "channel"])
    ap.add_argument("dims", help="n or nx,ny,nz voxels")
    ap.add_argument("modes", type=int)
    ap.add_argument("--radius", type=float, default=None, help="sphere obstacle radius in voxels")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None, help="write the basis here (.psfb)")
    a = ap.parse_args(argv)
    dims = tuple(int(x) for x in a.dims.split(","))
    dims = dims[0] if len(dims) == 1 else dims
    if a.kind == "sphere":
        dom = sphere_obstacle_domain(dims, a.radius if a.radius is not None else 0.25 * min(np.atleast_1d(dims)))
    elif a.kind == "channel":
        dom = channel_domain(dims if isinstance(dims, tuple) else (dims,) * 3)
    else:
        dom = box_domain(dims)
    b, stats = build_basis(dom, a.modes, device=a.device)
    if a.out:
        b.save(a.out)
    print(json.dumps({"domain": dom.name, "modes": a.modes,
                      **{k: (float(v) if isinstance(v, (float, np.floating)) else v) for k, v in stats.items()}}))


if __name__ == "__main__":
    main()
