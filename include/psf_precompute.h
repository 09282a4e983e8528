/*
 * psf_precompute.h -- C ABI of the per-domain precompute kernels: the
 * operator products of the Laplacian eigen-solve and the wedge -> advection
 * tensor build.
 *
 * Replaces the precompute half of the reference's solver set-up,
 * `PSFSolver::buildLaplace` and `PSFSolver::buildAdvection`
 * (Solver/SolverImpl/psfsolver.cpp:236-342 and :431-551, with the DEC
 * operators of DEC/dec.cpp:5-197 and :351-456), which assemble the pruned
 * 1-form Laplacian, run a shift-invert Arnoldi solver (Spectra) on the host,
 * and accumulate the advection tensor through dense E x N wedge matrices per
 * mode (O(N^2 E) doubles).  Here:
 *
 *  - the eigen-solve is Chebyshev-filtered subspace iteration on the
 *    symmetric interior operator K = (1/2h) d1_I^T *1dual d1_I (the pruned
 *    matrix of psfsolver.cpp:247-265 restricted to its non-zero rows); its
 *    operator product is psf_pre_csr_cheb, one fused kernel per polynomial
 *    degree.  The host side (Rayleigh-Ritz, QR) is
 *    parallelspectralfluids3d_b200/precompute.py;
 *  - the tensor C[k][a][j] = (1/lambda_k) sum_e Psi[e][a] W_k[e][j] with
 *    W_k[e][j] = sum_{f,g} S_e[f][g] Phi[f][k] Phi[g][j] (the wedge terms of
 *    psfsolver.cpp:520-533 gathered per edge into an antisymmetric 8 x 8
 *    matrix S_e over the faces its terms name) is psf_pre_advection_tensor:
 *    W is generated for a batch of k on the device and contracted with Psi
 *    by a split-K FP64 GEMM, reduced in a fixed order (deterministic).
 *
 * All arrays are device arrays on the current device; calls are enqueued on
 * `stream` (a cudaStream_t, 0 for the legacy default stream).  Every entry
 * point returns PSF_OK or a negative PSF_ERR_* code (psf_b200.h) and never
 * throws or exits.
 */
#ifndef PSF_PRECOMPUTE_H
#define PSF_PRECOMPUTE_H

#include "psf_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* out = alpha * (A Y) + beta * Y + gamma * X for a CSR matrix A (n_rows x
 * n_cols, int32 row pointers and column indices, FP64 values) and blocks of
 * m columns stored row-major with row stride `ld` doubles (ld even, m <= ld):
 * Y is n_cols x ld, X and out are n_rows x ld.  Columns [m, round_up(m, 2))
 * are computed too; columns beyond that are not touched.  beta != 0 needs a
 * square A; X is read only when gamma != 0.  The Chebyshev three-term
 * recurrence of the filtered subspace iteration is this call with
 * (alpha, beta, gamma) = (2 s / e, -2 s c / e, -s s_prev).  `out` must not
 * alias Y or X.  Replaces the sparse products inside the reference's
 * eigen-solve (psfsolver.cpp:277-281, Spectra's SparseGenRealShiftSolve). */
int psf_pre_csr_cheb(int64_t n_rows, int64_t n_cols, int32_t m, int64_t ld, const int32_t *row_ptr,
                     const int32_t *col_idx, const double *vals, const double *Y, const double *X, double *out,
                     double alpha, double beta, double gamma, void *stream);

/* Wedge data of a domain (built on the host from the voxels' 12 wedge terms,
 * psfsolver.cpp:456-533): for each of n_edges edges with terms, the rows in
 * `phi` of the faces its terms name (at most 8: an edge takes at most four
 * terms, and the reference's edge slots pair some terms with a face that does
 * not touch the edge), phi_zero_row for an empty slot; its antisymmetric S_e
 * (8 x 8, row-major, FP64); and its curl row Psi[e] (psfsolver.cpp:252, 342).
 * Columns are padded to `ldn`, a multiple of 128 that is >= n_modes, with
 * zeros. */
#define PSF_WEDGE_SLOTS 8

typedef struct psf_wedge_desc {
    int64_t n_edges;
    int32_t n_modes;
    int32_t ldn;
    const int32_t *edge_faces;  /* [n_edges][PSF_WEDGE_SLOTS] rows of phi */
    const double *edge_S;       /* [n_edges][PSF_WEDGE_SLOTS][PSF_WEDGE_SLOTS] */
    const double *psi;          /* [n_edges][ldn] */
    const double *phi;          /* [rows][ldn], row phi_zero_row all zero */
    int64_t phi_zero_row;
    const double *eigenvalues;  /* [n_modes] */
} psf_wedge_desc;

/* Device workspace bytes psf_pre_advection_tensor needs for a batch of
 * `k_batch` modes per pass (0 < k_batch <= min(n_modes, 64)). */
int psf_pre_advection_workspace(const psf_wedge_desc *d, int32_t k_batch, int64_t *bytes);

/* C[k][a][j] (FP64, [n_modes][n_modes][n_modes], device) of
 * psfsolver.cpp:539-550: C[k] = (1/lambda_k) Psi^T W_k.  `workspace` holds
 * at least psf_pre_advection_workspace(d, k_batch) bytes. */
int psf_pre_advection_tensor(const psf_wedge_desc *d, int32_t k_batch, void *workspace, int64_t workspace_bytes,
                             double *C, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PSF_PRECOMPUTE_H */
