// Single-instance step kernels with TMA staging: the contraction + FP64 state
// update and the reconstruction of the plain (FP32 basis) path as persistent
// kernels whose operand tiles arrive in shared memory by tensor-memory-access
// copies (cp.async.bulk.tensor, no multicast).
//
//   psf_contract_tma     C[k][a][j] as tiles of 32 rows (a) x 64 columns (j)
//                        of one k; threads form FP32 row dots with w_j from
//                        shared memory, scale them by w_a in FP64, and every
//                        tile leaves one FP64 partial dwpart[k][row chunk].
//                        The last CTA to finish (atomic ticket, no spinning)
//                        applies the FP64 update in the reference's order
//                        (psfsolver.cpp:37-59).
//                        (replaces simulation.cl:207-311, 356-394)
//   psf_reconstruct_tma  Phi^T[i][f] as tiles of 64 faces x 64 modes; a tile's
//                        64 faces are summed over all modes in FP32, then
//                        written to the reference face numbering and to the
//                        face-pair field.  (replaces simulation.cl:313-354)
//
// One producer warp issues the copies into a ring of stages; eight consumer
// warps wait on each stage's mbarrier, compute, and release it.  Every wait
// is bounded (psf_sm100.cuh): a wait that gives up records a code in the
// context's error word.  A consumer warp whose wait gave up stops waiting but
// keeps walking the same tiles and named barriers as the others, so no
// barrier is left short; the producer waits (bounded) for the copies it still
// has in flight before the CTA exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "psf_b200.h"
#include "psf_internal.h"
#include "psf_plain_tma.h"
#include "psf_sm100.cuh"

namespace psf {

using namespace sm100;

namespace {

constexpr int CONSUMERS = 256;           // eight consumer warps
constexpr int THREADS = CONSUMERS + 32;  // plus one producer warp

__device__ __forceinline__ void consumer_bar() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// FP64 sum over the 256 consumer threads (fixed order: warp shuffles, then warps 0..7).
__device__ __forceinline__ double consumer_sum(double v, double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    consumer_bar();
    if (lane == 0) red[warp] = v;
    consumer_bar();
    double t = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) t += red[i];
    return t;
}

// Producer loop shared by both kernels: `ks_per_tile` copies per tile, each
// started by `issue(stage, bar, tile, ks)`.
template <int STAGES, class Issue>
__device__ __forceinline__ void produce(uint64_t *full, uint64_t *empty, int n_tiles, int ks_per_tile,
                                        uint32_t stage_bytes, int *err, Issue issue)
{
    uint32_t last_parity[STAGES];
    bool issued[STAGES];
#pragma unroll
    for (int s = 0; s < STAGES; ++s) issued[s] = false;
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int t = blockIdx.x; ok && t < n_tiles; t += gridDim.x) {
        for (int ks = 0; ks < ks_per_tile; ++ks) {
            if (!mbar_wait(&empty[stage], phase ^ 1u, err, ERR_WAIT_EMPTY)) {
                ok = false;
                break;
            }
            mbar_arrive_expect_tx(&full[stage], stage_bytes);
            issue(stage, &full[stage], t, ks);
            issued[stage] = true;
            last_parity[stage] = phase;
            if (++stage == STAGES) {
                stage = 0;
                phase ^= 1u;
            }
        }
    }
    // After an error, copies may still be in flight that no one consumes:
    // wait (bounded) for them before the CTA exits.
    if (*(volatile int *)err != 0)
        for (int s = 0; s < STAGES; ++s)
            if (issued[s]) mbar_wait(&full[s], last_parity[s], err, ERR_WAIT_DRAIN);
}

constexpr int CT_ROWS = 32, CT_COLS = 64, CT_STAGES = 12;
constexpr uint32_t CT_STAGE_BYTES = CT_ROWS * CT_COLS * 4;
constexpr int RT_FACES = 64, RT_MODES = 64, RT_STAGES = 8;
constexpr uint32_t RT_STAGE_BYTES = RT_FACES * RT_MODES * 4;

}  // namespace

// ------------------------------------------------------------ contraction
__global__ void __launch_bounds__(THREADS, 1) psf_contract_tma(const __grid_constant__ CUtensorMap tmC, int N, int KC,
                                                               int RC, double *__restrict__ w,
                                                               double *__restrict__ dwpart,
                                                               const double *__restrict__ lam,
                                                               const double *__restrict__ force, StateParams sp,
                                                               unsigned int *__restrict__ ticket,
                                                               unsigned long long *__restrict__ step_ctr, int *err)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    float *stages = reinterpret_cast<float *>(smem);                           // [STAGES][32 rows][64 columns]
    float *wj = reinterpret_cast<float *>(smem + CT_STAGES * CT_STAGE_BYTES);  // [KC * 64]
    double *wd = reinterpret_cast<double *>(wj + KC * CT_COLS);                // [RC * 32]
    double *red = wd + RC * CT_ROWS;                                           // [8]
    double *wnew = red + 8;                                                    // [N] (last CTA)
    uint64_t *full = reinterpret_cast<uint64_t *>(wnew + ((N + 1) & ~1));
    uint64_t *empty = full + CT_STAGES;
    __shared__ int is_last, cta_ok;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_tiles = N * RC;
    if (threadIdx.x == 0) {
        for (int s = 0; s < CT_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 8);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (warp == 8) {
        if (lane == 0) {
            tma_prefetch_desc(&tmC);
            produce<CT_STAGES>(full, empty, n_tiles, KC, CT_STAGE_BYTES, err, [&](int s, uint64_t *bar, int t, int ks) {
                const int k = t / RC, rc = t - k * RC;
                tma_load_3d(stages + (size_t)s * CT_ROWS * CT_COLS, &tmC, bar, ks * CT_COLS, rc * CT_ROWS, k);
            });
        }
        return;
    }
    // w in shared memory: FP32 columns (zero beyond N) and FP64 rows.
    for (int i = threadIdx.x; i < KC * CT_COLS; i += CONSUMERS) wj[i] = i < N ? (float)w[i] : 0.f;
    for (int i = threadIdx.x; i < RC * CT_ROWS; i += CONSUMERS) wd[i] = i < N ? w[i] : 0.0;
    if (threadIdx.x == 0) cta_ok = 1;
    consumer_bar();
    // Thread (r, cg): row r of the tile, columns cg*4..+3 and 32+cg*4..+3 of each stage.
    const int r = threadIdx.x >> 3, cg = threadIdx.x & 7;
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const int k = t / RC, rc = t - k * RC;
        float part = 0.f;
        for (int ks = 0; ks < KC; ++ks) {
            if (ok && !mbar_wait(&full[stage], phase, err, ERR_WAIT_FULL)) ok = false;
            if (ok) {
                const float *row = stages + (size_t)stage * CT_ROWS * CT_COLS + r * CT_COLS;
                const float4 v0 = *reinterpret_cast<const float4 *>(row + cg * 4);
                const float4 v1 = *reinterpret_cast<const float4 *>(row + 32 + cg * 4);
                const float *wc = wj + ks * CT_COLS;
                part = fmaf(v0.x, wc[cg * 4 + 0], part);
                part = fmaf(v0.y, wc[cg * 4 + 1], part);
                part = fmaf(v0.z, wc[cg * 4 + 2], part);
                part = fmaf(v0.w, wc[cg * 4 + 3], part);
                part = fmaf(v1.x, wc[32 + cg * 4 + 0], part);
                part = fmaf(v1.y, wc[32 + cg * 4 + 1], part);
                part = fmaf(v1.z, wc[32 + cg * 4 + 2], part);
                part = fmaf(v1.w, wc[32 + cg * 4 + 3], part);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[stage]);
            if (++stage == CT_STAGES) {
                stage = 0;
                phase ^= 1u;
            }
        }
        const double acc = wd[rc * CT_ROWS + r] * (double)part;
        const double tot = consumer_sum(acc, red);
        if (threadIdx.x == 0) dwpart[(size_t)k * RC + rc] = tot;
    }
    if (!ok) cta_ok = 0;
    consumer_bar();
    // A CTA whose waits gave up leaves the ticket alone: the step is abandoned
    // and the host reads the error word.
    if (threadIdx.x == 0) {
        is_last = 0;
        if (cta_ok) {
            __threadfence();
            const unsigned int prev = atomicAdd(ticket, 1u);
            is_last = (prev == gridDim.x - 1);
        }
    }
    consumer_bar();
    if (!is_last) return;
    __threadfence();

    // Last CTA: FP64 state update in the reference's order (psfsolver.cpp:37-59).
    double e1 = 0.0, e2 = 0.0;
    for (int i = threadIdx.x; i < N; i += CONSUMERS) {
        const double wi = w[i];
        double dw = 0.0;
        for (int q = 0; q < RC; ++q) dw += __ldcg(dwpart + (size_t)i * RC + q);
        const double w1 = wi + sp.dt * dw;
        wnew[i] = w1;
        e1 += wi * wi;
        e2 += w1 * w1;
    }
    e1 = consumer_sum(e1, red);
    e2 = consumer_sum(e2, red);
    const double scale = (sp.flags & PSF_FLAG_RENORM) ? sqrt(e1 / e2) : 1.0;
    for (int i = threadIdx.x; i < N; i += CONSUMERS) {
        double v = wnew[i] * scale;
        v *= exp(sp.visc_signed * lam[i] * sp.dt);
        if (sp.flags & PSF_FLAG_FORCING) v += sp.dt * force[i];
        w[i] = v;
    }
    if (threadIdx.x == 0) {
        *ticket = 0u;
        *step_ctr += 1ull;
    }
}

// --------------------------------------------------------- reconstruction
__global__ void __launch_bounds__(THREADS, 1) psf_reconstruct_tma(const __grid_constant__ CUtensorMap tmP, int N,
                                                                  int KS, long long n_active,
                                                                  const double *__restrict__ w,
                                                                  const int32_t *__restrict__ faces,
                                                                  float *__restrict__ u, float *__restrict__ pairs,
                                                                  const int32_t *__restrict__ pair_dst, int *err)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    float *stages = reinterpret_cast<float *>(smem);                           // [STAGES][64 modes][64 faces]
    float *wsm = reinterpret_cast<float *>(smem + RT_STAGES * RT_STAGE_BYTES); // [KS * 64]
    float *red = wsm + KS * RT_MODES;                                          // [4][64]
    uint64_t *full = reinterpret_cast<uint64_t *>(red + 4 * RT_FACES);
    uint64_t *empty = full + RT_STAGES;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_tiles = (int)((n_active + RT_FACES - 1) / RT_FACES);
    if (threadIdx.x == 0) {
        for (int s = 0; s < RT_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 8);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (warp == 8) {
        if (lane == 0) {
            tma_prefetch_desc(&tmP);
            produce<RT_STAGES>(full, empty, n_tiles, KS, RT_STAGE_BYTES, err, [&](int s, uint64_t *bar, int t, int ks) {
                tma_load_2d(stages + (size_t)s * RT_FACES * RT_MODES, &tmP, bar, t * RT_FACES, ks * RT_MODES);
            });
        }
        return;
    }
    for (int i = threadIdx.x; i < KS * RT_MODES; i += CONSUMERS) wsm[i] = i < N ? (float)w[i] : 0.f;
    consumer_bar();
    // Thread (g, f): face f of the tile, modes g*16..g*16+15 of every stage.
    const int f = threadIdx.x & 63, g = threadIdx.x >> 6;
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        float acc = 0.f;
        for (int ks = 0; ks < KS; ++ks) {
            if (ok && !mbar_wait(&full[stage], phase, err, ERR_WAIT_FULL)) ok = false;
            if (ok) {
                const float *st = stages + (size_t)stage * RT_FACES * RT_MODES + (g * 16) * RT_FACES + f;
                const float *wm = wsm + ks * RT_MODES + g * 16;
#pragma unroll
                for (int m = 0; m < 16; ++m) acc = fmaf(st[m * RT_FACES], wm[m], acc);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[stage]);
            if (++stage == RT_STAGES) {
                stage = 0;
                phase ^= 1u;
            }
        }
        red[g * RT_FACES + f] = acc;
        consumer_bar();
        if (ok && threadIdx.x < RT_FACES) {
            const long long r = (long long)t * RT_FACES + threadIdx.x;
            if (r < n_active) {
                const float v = (red[threadIdx.x] + red[RT_FACES + threadIdx.x]) +
                                (red[2 * RT_FACES + threadIdx.x] + red[3 * RT_FACES + threadIdx.x]);
                u[faces[r]] = v;
                const int32_t d0 = pair_dst[2 * r], d1 = pair_dst[2 * r + 1];
                if (d0 >= 0) pairs[d0] = v;
                if (d1 >= 0) pairs[d1] = v;
            }
        }
        consumer_bar();
    }
}

// ---------------------------------------------------------------- host
int contract_tma_row_chunks(int N) { return (N + CT_ROWS - 1) / CT_ROWS; }

int contract_tma_smem_bytes(int N)
{
    const int KC = (N + CT_COLS - 1) / CT_COLS, RC = contract_tma_row_chunks(N);
    return CT_STAGES * (int)CT_STAGE_BYTES + KC * CT_COLS * 4 + RC * CT_ROWS * 8 + 8 * 8 + ((N + 1) & ~1) * 8 +
           2 * CT_STAGES * 8;
}

int reconstruct_tma_smem_bytes(int N)
{
    const int KS = (N + RT_MODES - 1) / RT_MODES;
    return RT_STAGES * (int)RT_STAGE_BYTES + KS * RT_MODES * 4 + 4 * RT_FACES * 4 + 2 * RT_STAGES * 8;
}

int make_plain_tma_maps(const PlainDev &d, CUtensorMap *tmC, CUtensorMap *tmP)
{
    // C: [k][a][j] FP32, j padded to Np (a multiple of 4: 16-byte rows).
    const uint64_t dc[3] = {(uint64_t)d.Np, (uint64_t)d.N, (uint64_t)d.N};
    const uint64_t sc[2] = {(uint64_t)d.Np * 4, (uint64_t)d.N * d.Np * 4};
    const uint32_t bc[3] = {CT_COLS, CT_ROWS, 1};
    int rc = encode_tensor_map_f32(tmC, const_cast<float *>(d.C), 3, dc, sc, bc);
    if (rc != PSF_OK) return rc;
    // Phi^T: [i][f] FP32, f padded to ldp (a multiple of 4).
    const uint64_t dp[2] = {(uint64_t)d.ldp, (uint64_t)d.N};
    const uint64_t sp[1] = {(uint64_t)d.ldp * 4};
    const uint32_t bp[2] = {RT_FACES, RT_MODES};
    return encode_tensor_map_f32(tmP, const_cast<float *>(d.phiT), 2, dp, sp, bp);
}

// The dynamic shared-memory limit is a per-device attribute of each kernel;
// it is raised once per device to what N = PSF_MAX_MODES needs.
template <class K>
static int configure_smem(K kernel, int bytes, unsigned long long &configured)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured & bit)) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        configured |= bit;
    }
    return PSF_OK;
}

int launch_contract_tma(const PlainDev &d, const CUtensorMap &tmC, int grid, int *err, cudaStream_t st)
{
    static unsigned long long configured = 0;
    int rc = configure_smem(psf_contract_tma, contract_tma_smem_bytes(PSF_MAX_MODES), configured);
    if (rc != PSF_OK) return rc;
    const int KC = (d.N + CT_COLS - 1) / CT_COLS, RC = contract_tma_row_chunks(d.N);
    const int g = std::max(1, std::min(grid, d.N * RC));
    psf_contract_tma<<<g, THREADS, contract_tma_smem_bytes(d.N), st>>>(tmC, d.N, KC, RC, d.w, d.dwpart, d.lam,
                                                                       d.force, d.sp, d.ticket, d.step_ctr, err);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_contract_tma launch");
}

int launch_reconstruct_tma(const PlainDev &d, const CUtensorMap &tmP, int grid, int *err, cudaStream_t st)
{
    static unsigned long long configured = 0;
    int rc = configure_smem(psf_reconstruct_tma, reconstruct_tma_smem_bytes(PSF_MAX_MODES), configured);
    if (rc != PSF_OK) return rc;
    const int KS = (d.N + RT_MODES - 1) / RT_MODES;
    const long long tiles = (d.n_active + RT_FACES - 1) / RT_FACES;
    const int g = (int)std::max<long long>(1, std::min<long long>(grid, tiles));
    psf_reconstruct_tma<<<g, THREADS, reconstruct_tma_smem_bytes(d.N), st>>>(
        tmP, d.N, KS, d.n_active, d.w, d.faces, d.u, reinterpret_cast<float *>(d.pairs), d.pair_dst, err);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_reconstruct_tma launch");
}

}  // namespace psf
