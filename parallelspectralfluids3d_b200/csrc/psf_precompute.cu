// Per-domain precompute kernels (include/psf_precompute.h): the operator
// product of the eigen-solve and the advection tensor build, FP64 throughout.
//
//   psf_csr_cheb     one warp per row of a CSR matrix, 16-byte gathers of the
//                    block's rows, fused with the Chebyshev three-term
//                    recurrence (out = alpha A Y + beta Y + gamma X)
//   psf_wedge_w      W[e][kk][j] = sum_g q_e[g][kk] Phi[g_e][j] with
//                    q_e[g][kk] = sum_f S_e[f][g] Phi[f_e][k0 + kk] over the
//                    (at most 8) faces the edge's terms name: the wedge
//                    matrices of a batch of modes, one warp per edge
//   psf_wedge_gemm   partial[s][a][c] = sum_{e in split s} Psi[e][a] W[e][c]:
//                    a 128 x 128 x 16 FP64 tile GEMM with a three-stage
//                    cp.async pipeline, split along the edges
//   psf_wedge_reduce C[k][a][j] = (1/lambda_k) sum_s partial[s][a][kk ldn + j],
//                    splits summed in a fixed order (deterministic)
//
// The reference builds the same tensor with dense E x N matrices per mode
// (Solver/SolverImpl/psfsolver.cpp:431-551); here the 12 wedge terms of every
// voxel are gathered per edge into an antisymmetric matrix over the faces
// its terms name, so W_k is generated on the fly from Phi and never held for
// more than a batch of modes.  (The reference's edge slots pair one term in
// twelve with a face that does not touch the edge, so an edge can name five
// faces; eight slots cover any four terms.)

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "psf_internal.h"
#include "psf_precompute.h"

namespace {

using psf::cuda_fail;
using psf::fail;

// ------------------------------------------------------------- CSR x block
// Warp w of the grid takes rows w, w + warps, ...; the row's non-zeros are
// staged in the warp's shared slots (broadcast reads), and lane l owns the
// double2 columns l, l + 32, ... of the block.
__global__ void __launch_bounds__(256) psf_csr_cheb(long long n_rows, int m2, long long ld2,
                                                    const int32_t *__restrict__ row_ptr,
                                                    const int32_t *__restrict__ col_idx,
                                                    const double *__restrict__ vals, const double2 *__restrict__ Y,
                                                    const double2 *__restrict__ X, double2 *__restrict__ out,
                                                    double alpha, double beta, double gamma)
{
    __shared__ int32_t scol[8][32];
    __shared__ double sval[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long nwarps = (long long)gridDim.x * 8;
    for (long long row = (long long)blockIdx.x * 8 + warp; row < n_rows; row += nwarps) {
        const int b = __ldg(row_ptr + row), e = __ldg(row_ptr + row + 1);
        for (int c0 = 0; c0 < m2; c0 += 32) {
            const int c = c0 + lane;
            double2 acc = make_double2(0.0, 0.0);
            for (int p0 = b; p0 < e; p0 += 32) {
                const int cnt = min(32, e - p0);
                __syncwarp();
                if (lane < cnt) {
                    scol[warp][lane] = __ldg(col_idx + p0 + lane);
                    sval[warp][lane] = __ldg(vals + p0 + lane);
                }
                __syncwarp();
                if (c < m2) {
                    int q = 0;
                    for (; q + 4 <= cnt; q += 4) {
                        const double2 y0 = __ldg(Y + (size_t)scol[warp][q] * ld2 + c);
                        const double2 y1 = __ldg(Y + (size_t)scol[warp][q + 1] * ld2 + c);
                        const double2 y2 = __ldg(Y + (size_t)scol[warp][q + 2] * ld2 + c);
                        const double2 y3 = __ldg(Y + (size_t)scol[warp][q + 3] * ld2 + c);
                        const double v0 = sval[warp][q], v1 = sval[warp][q + 1];
                        const double v2 = sval[warp][q + 2], v3 = sval[warp][q + 3];
                        acc.x = fma(v0, y0.x, acc.x);
                        acc.y = fma(v0, y0.y, acc.y);
                        acc.x = fma(v1, y1.x, acc.x);
                        acc.y = fma(v1, y1.y, acc.y);
                        acc.x = fma(v2, y2.x, acc.x);
                        acc.y = fma(v2, y2.y, acc.y);
                        acc.x = fma(v3, y3.x, acc.x);
                        acc.y = fma(v3, y3.y, acc.y);
                    }
                    for (; q < cnt; ++q) {
                        const double2 y = __ldg(Y + (size_t)scol[warp][q] * ld2 + c);
                        const double v = sval[warp][q];
                        acc.x = fma(v, y.x, acc.x);
                        acc.y = fma(v, y.y, acc.y);
                    }
                }
            }
            if (c < m2) {
                double2 r = make_double2(alpha * acc.x, alpha * acc.y);
                if (beta != 0.0) {
                    const double2 y = __ldg(Y + (size_t)row * ld2 + c);
                    r.x = fma(beta, y.x, r.x);
                    r.y = fma(beta, y.y, r.y);
                }
                if (gamma != 0.0) {
                    const double2 x = __ldg(X + (size_t)row * ld2 + c);
                    r.x = fma(gamma, x.x, r.x);
                    r.y = fma(gamma, x.y, r.y);
                }
                out[(size_t)row * ld2 + c] = r;
            }
        }
    }
}

// ------------------------------------------------------------ wedge terms
constexpr int WEDGE_KB_MAX = 64;  // modes per W batch (shared-memory q table)
constexpr int SLOTS = PSF_WEDGE_SLOTS;

// One warp per edge: q_e[g][kk] in shared memory (used slots compacted to
// the front), then the edge's W rows.  Slots holding the zero row are
// skipped; the test is warp-uniform.  Rows e >= n_edges (padding up to whole
// GEMM chunks) are written as zeros.
__global__ void __launch_bounds__(256) psf_wedge_w(long long n_edges, long long n_rows, int ldn, int k0, int kb,
                                                   const int32_t *__restrict__ edge_faces,
                                                   const double *__restrict__ edge_S,
                                                   const double *__restrict__ phi, long long zero_row,
                                                   double *__restrict__ W)
{
    __shared__ double qs[8][SLOTS][WEDGE_KB_MAX];
    __shared__ int32_t fs[8][SLOTS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long nwarps = (long long)gridDim.x * 8;
    const int ld2 = ldn / 2;
    for (long long e = (long long)blockIdx.x * 8 + warp; e < n_rows; e += nwarps) {
        double2 *We = reinterpret_cast<double2 *>(W + (size_t)e * kb * ldn);
        if (e >= n_edges) {
            for (int i = lane; i < kb * ld2; i += 32) We[i] = make_double2(0.0, 0.0);
            continue;
        }
        __syncwarp();
        int f[SLOTS];
#pragma unroll
        for (int g = 0; g < SLOTS; ++g) f[g] = __ldg(edge_faces + (size_t)SLOTS * e + g);
        for (int kk = lane; kk < kb; kk += 32) {
            double pk[SLOTS];
#pragma unroll
            for (int h = 0; h < SLOTS; ++h)
                pk[h] = f[h] == zero_row ? 0.0 : __ldg(phi + (size_t)f[h] * ldn + k0 + kk);
            int u = 0;
#pragma unroll
            for (int g = 0; g < SLOTS; ++g) {
                if (f[g] == zero_row) continue;
                double q = 0.0;
#pragma unroll
                for (int h = 0; h < SLOTS; ++h) q = fma(__ldg(edge_S + ((size_t)SLOTS * e + h) * SLOTS + g), pk[h], q);
                qs[warp][u++][kk] = q;
            }
        }
        int used = 0;
#pragma unroll
        for (int g = 0; g < SLOTS; ++g)
            if (f[g] != zero_row) {
                if (lane == 0) fs[warp][used] = f[g];
                ++used;
            }
        __syncwarp();
        for (int j2 = lane; j2 < ld2; j2 += 32) {
            double2 p[SLOTS];
#pragma unroll
            for (int g = 0; g < SLOTS; ++g)
                if (g < used) p[g] = __ldg(reinterpret_cast<const double2 *>(phi + (size_t)fs[warp][g] * ldn) + j2);
            for (int kk = 0; kk < kb; ++kk) {
                double2 w = make_double2(0.0, 0.0);
#pragma unroll
                for (int g = 0; g < SLOTS; ++g)
                    if (g < used) {
                        const double q = qs[warp][g][kk];
                        w.x = fma(q, p[g].x, w.x);
                        w.y = fma(q, p[g].y, w.y);
                    }
                We[(size_t)kk * ld2 + j2] = w;
            }
        }
    }
}

// ---------------------------------------------------------- FP64 tile GEMM
constexpr int GB_M = 128, GB_N = 128, GB_K = 16, GB_STAGES = 3, GB_THREADS = 256;
constexpr int GB_SMEM = GB_STAGES * GB_K * (GB_M + GB_N) * 8;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// partial[split][a][c] over the edge chunks [chunk0, chunk1) of split
// `blockIdx.z`: A = psi [n_edges][ldn] (rows beyond n_edges read as zero),
// B = W [rows][ldc].  Thread (ty, tx) owns rows a0 + 2 ty + 32 i + {0,1} and
// columns c0 + 2 tx + 32 j + {0,1} (i, j < 4): conflict-free 16-byte
// shared-memory reads (A broadcast within a warp, B contiguous).
__global__ void __launch_bounds__(GB_THREADS, 1) psf_wedge_gemm(long long n_edges, int ldn, long long ldc,
                                                               long long chunks_per_split, long long n_chunks,
                                                               const double *__restrict__ psi,
                                                               const double *__restrict__ W,
                                                               double *__restrict__ partial)
{
    extern __shared__ __align__(16) double gsm[];
    double *As = gsm;                            // [STAGES][K][M]
    double *Bs = gsm + GB_STAGES * GB_K * GB_M;  // [STAGES][K][N]
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    const int a0 = blockIdx.y * GB_M;
    const long long c0 = (long long)blockIdx.x * GB_N;
    const long long ch0 = (long long)blockIdx.z * chunks_per_split;
    const long long ch1 = min(n_chunks, ch0 + chunks_per_split);
    const long long nk = max(0ll, ch1 - ch0);

    auto load_stage = [&](long long kt, int slot) {
        const long long e0 = (ch0 + kt) * GB_K;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int q = tid + GB_THREADS * r;  // 1024 16-byte pieces per operand tile
            const int row = q >> 6, piece = q & 63;
            const long long e = e0 + row;
            const bool ok = e < n_edges;
            const double *srcA = ok ? psi + (size_t)e * ldn + a0 + 2 * piece : psi;
            cp_async16(As + ((size_t)slot * GB_K + row) * GB_M + 2 * piece, srcA, ok ? 16 : 0);
            const double *srcB = W + (size_t)e * ldc + c0 + 2 * piece;
            cp_async16(Bs + ((size_t)slot * GB_K + row) * GB_N + 2 * piece, srcB, 16);
        }
    };

    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;

#pragma unroll
    for (int s = 0; s < GB_STAGES - 1; ++s) {
        if (s < nk) load_stage(s, s);
        cp_async_commit();
    }
    for (long long kt = 0; kt < nk; ++kt) {
        cp_async_wait<GB_STAGES - 2>();
        __syncthreads();
        const long long nxt = kt + GB_STAGES - 1;
        if (nxt < nk) load_stage(nxt, (int)(nxt % GB_STAGES));
        cp_async_commit();
        const int slot = (int)(kt % GB_STAGES);
        const double *A = As + (size_t)slot * GB_K * GB_M;
        const double *B = Bs + (size_t)slot * GB_K * GB_N;
#pragma unroll
        for (int kk = 0; kk < GB_K; ++kk) {
            double a[8], b[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double2 v = *reinterpret_cast<const double2 *>(A + kk * GB_M + 2 * ty + 32 * i);
                a[2 * i] = v.x;
                a[2 * i + 1] = v.y;
                const double2 u = *reinterpret_cast<const double2 *>(B + kk * GB_N + 2 * tx + 32 * i);
                b[2 * i] = u.x;
                b[2 * i + 1] = u.y;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
    }
    cp_async_wait<0>();

    double *P = partial + (size_t)blockIdx.z * ldn * ldc;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int ii = 0; ii < 2; ++ii) {
            const int a = a0 + 2 * ty + 32 * i + ii;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const long long c = c0 + 2 * tx + 32 * j;
                *reinterpret_cast<double2 *>(P + (size_t)a * ldc + c) =
                    make_double2(acc[2 * i + ii][2 * j], acc[2 * i + ii][2 * j + 1]);
            }
        }
}

__global__ void psf_wedge_reduce(int N, int ldn, long long ldc, int k0, int kb, int splits,
                                 const double *__restrict__ partial, const double *__restrict__ lam,
                                 double *__restrict__ C)
{
    const long long total = (long long)kb * N * N;
    const size_t split_stride = (size_t)ldn * ldc;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t % N);
        const int a = (int)((t / N) % N);
        const int kk = (int)(t / ((long long)N * N));
        const size_t src = (size_t)a * ldc + (size_t)kk * ldn + j;
        double s = 0.0;
        for (int p = 0; p < splits; ++p) s += partial[p * split_stride + src];
        const int k = k0 + kk;
        C[((size_t)k * N + a) * N + j] = s / lam[k];
    }
}

// Work split of one W batch: GEMM tiles per batch and the number of edge
// splits that gives the grid about two tiles per SM.
struct WedgePlan {
    long long n_chunks, rows, ldc, tiles, splits, chunks_per_split;
    size_t w_bytes, partial_bytes;
};

WedgePlan plan_of(const psf_wedge_desc *d, int kb)
{
    WedgePlan p{};
    p.n_chunks = (d->n_edges + GB_K - 1) / GB_K;
    p.rows = p.n_chunks * GB_K;
    p.ldc = (long long)kb * d->ldn;
    p.tiles = (long long)(d->ldn / GB_M) * (p.ldc / GB_N);
    const long long want = std::max(1ll, (2ll * 148 + p.tiles - 1) / p.tiles);
    p.splits = std::max(1ll, std::min({want, 64ll, std::max(1ll, p.n_chunks)}));
    p.chunks_per_split = std::max(1ll, (p.n_chunks + p.splits - 1) / p.splits);
    p.splits = std::max(1ll, (p.n_chunks + p.chunks_per_split - 1) / p.chunks_per_split);
    p.w_bytes = (size_t)p.rows * p.ldc * sizeof(double);
    p.partial_bytes = (size_t)p.splits * d->ldn * p.ldc * sizeof(double);
    return p;
}

// Workspace layout: W of a full batch at offset 0, then the partial sums,
// sized for the larger of the full batch and the last (shorter) one, whose
// edge split may differ.
struct Workspace {
    size_t w_bytes, partial_bytes;
};

Workspace workspace_of(const psf_wedge_desc *d, int kb)
{
    const WedgePlan full = plan_of(d, kb);
    size_t partial = full.partial_bytes;
    const int last = d->n_modes % kb;
    if (last) partial = std::max(partial, plan_of(d, last).partial_bytes);
    return Workspace{full.w_bytes, partial};
}

int check_desc(const psf_wedge_desc *d, int kb)
{
    if (!d) return fail(PSF_ERR_INVALID, "null wedge descriptor");
    if (d->n_edges < 0 || d->n_modes < 1 || d->ldn < d->n_modes || d->ldn % GB_M != 0)
        return fail(PSF_ERR_INVALID, "wedge descriptor: n_modes >= 1 and ldn a multiple of 128 >= n_modes");
    if (kb < 1 || kb > d->n_modes || kb > WEDGE_KB_MAX)
        return fail(PSF_ERR_INVALID, "k_batch must be in [1, min(n_modes, 64)]");
    if (d->n_edges > 0 && (!d->edge_faces || !d->edge_S || !d->psi))
        return fail(PSF_ERR_INVALID, "null wedge array");
    if (!d->phi || !d->eigenvalues) return fail(PSF_ERR_INVALID, "null phi or eigenvalues");
    if (d->phi_zero_row < 0) return fail(PSF_ERR_INVALID, "phi_zero_row must be a row of phi");
    return PSF_OK;
}

}  // namespace

extern "C" int psf_pre_csr_cheb(int64_t n_rows, int64_t n_cols, int32_t m, int64_t ld, const int32_t *row_ptr,
                                const int32_t *col_idx, const double *vals, const double *Y, const double *X,
                                double *out, double alpha, double beta, double gamma, void *stream)
{
    if (n_rows < 0 || n_cols < 0 || m < 0 || ld < m || (ld & 1))
        return fail(PSF_ERR_INVALID, "psf_pre_csr_cheb: need 0 <= m <= ld, ld even");
    if (beta != 0.0 && n_rows != n_cols)
        return fail(PSF_ERR_INVALID, "psf_pre_csr_cheb: beta != 0 needs a square matrix");
    if (n_rows == 0 || m == 0) return PSF_OK;
    if (!row_ptr || !col_idx || !vals || !Y || !out || (gamma != 0.0 && !X))
        return fail(PSF_ERR_INVALID, "psf_pre_csr_cheb: null array");
    if ((reinterpret_cast<uintptr_t>(Y) | reinterpret_cast<uintptr_t>(out) |
         (gamma != 0.0 ? reinterpret_cast<uintptr_t>(X) : 0)) & 15)
        return fail(PSF_ERR_INVALID, "psf_pre_csr_cheb: blocks must be 16-byte aligned");
    if (out == Y || (gamma != 0.0 && out == X))
        return fail(PSF_ERR_INVALID, "psf_pre_csr_cheb: out aliases an input");
    const long long blocks = std::min<long long>((n_rows + 7) / 8, 148ll * 16);
    psf_csr_cheb<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        n_rows, (m + 1) / 2, ld / 2, row_ptr, col_idx, vals, reinterpret_cast<const double2 *>(Y),
        reinterpret_cast<const double2 *>(X), reinterpret_cast<double2 *>(out), alpha, beta, gamma);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_csr_cheb launch");
}

extern "C" int psf_pre_advection_workspace(const psf_wedge_desc *d, int32_t k_batch, int64_t *bytes)
{
    int rc = check_desc(d, k_batch);
    if (rc != PSF_OK) return rc;
    if (!bytes) return fail(PSF_ERR_INVALID, "null output");
    const Workspace ws = workspace_of(d, k_batch);
    *bytes = (int64_t)(ws.w_bytes + ws.partial_bytes);
    return PSF_OK;
}

extern "C" int psf_pre_advection_tensor(const psf_wedge_desc *d, int32_t k_batch, void *workspace,
                                        int64_t workspace_bytes, double *C, void *stream)
{
    int rc = check_desc(d, k_batch);
    if (rc != PSF_OK) return rc;
    if (!C || !workspace) return fail(PSF_ERR_INVALID, "null tensor or workspace");
    const Workspace ws = workspace_of(d, k_batch);
    if (workspace_bytes < 0 || (size_t)workspace_bytes < ws.w_bytes + ws.partial_bytes)
        return fail(PSF_ERR_INVALID, "workspace smaller than psf_pre_advection_workspace");
    if ((reinterpret_cast<uintptr_t>(workspace) | reinterpret_cast<uintptr_t>(d->psi) |
         reinterpret_cast<uintptr_t>(d->phi)) & 15)
        return fail(PSF_ERR_INVALID, "workspace, psi and phi must be 16-byte aligned");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double *W = static_cast<double *>(workspace);
    double *partial = reinterpret_cast<double *>(static_cast<char *>(workspace) + ws.w_bytes);
    static bool configured[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev >= 64 || !configured[dev]) {
        e = cudaFuncSetAttribute(psf_wedge_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, GB_SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(psf_wedge_gemm)");
        if (dev < 64) configured[dev] = true;
    }
    const int N = d->n_modes;
    for (int k0 = 0; k0 < N; k0 += k_batch) {
        const int kb = std::min(k_batch, N - k0);
        const WedgePlan q = plan_of(d, kb);
        const long long wblocks = std::max(1ll, std::min<long long>((q.rows + 7) / 8, 148ll * 16));
        psf_wedge_w<<<(unsigned)wblocks, 256, 0, st>>>(d->n_edges, q.rows, d->ldn, k0, kb, d->edge_faces, d->edge_S,
                                                       d->phi, d->phi_zero_row, W);
        if (q.n_chunks > 0) {
            const dim3 grid((unsigned)(q.ldc / GB_N), (unsigned)(d->ldn / GB_M), (unsigned)q.splits);
            psf_wedge_gemm<<<grid, GB_THREADS, GB_SMEM, st>>>(d->n_edges, d->ldn, q.ldc, q.chunks_per_split,
                                                             q.n_chunks, d->psi, W, partial);
        } else {
            e = cudaMemsetAsync(partial, 0, q.partial_bytes, st);
            if (e != cudaSuccess) return cuda_fail(e, "clearing the partial sums");
        }
        const long long total = (long long)kb * N * N;
        const long long rblocks = std::min<long long>((total + 255) / 256, 148ll * 32);
        psf_wedge_reduce<<<(unsigned)rblocks, 256, 0, st>>>(N, d->ldn, q.ldc, k0, kb, (int)q.splits, partial,
                                                           d->eigenvalues, C);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "advection tensor launch");
    }
    return PSF_OK;
}
