// Coefficient half of a single-instance step (FP32 basis) as ONE persistent,
// cooperative kernel with TMA staging (cp.async.bulk.tensor, no multicast):
//
//   1. contraction: tiles of 32 rows (a) x 64 columns (j) of one C_k; threads
//      form FP32 row dots with w_j, scale them by w_a in FP64, and every tile
//      leaves one FP64 partial dwpart[k][row chunk];
//   2. grid barrier (bounded);
//   3. every CTA applies the FP64 state update itself, from the partials and
//      its own shared-memory copy of w^n, in the reference's order
//      (psfsolver.cpp:37-59); CTA 0 publishes w^{n+1};
//   4. reconstruction u = Phi w^{n+1}: tiles of 64 faces x 64 modes of Phi
//      (stored tile by tile, so each copy is 16 KB of contiguous memory),
//      summed in FP32 and written to the reference face numbering and to the
//      per-voxel face-pair field the tracer reads.
//   (replaces simulation.cl:207-394: advection_reduce_x/y, energy,
//    update_vel, normalization_viscocity_gravity, reconstruct_velocity_field)
//
// A producer warp streams the C tiles and then the Phi tiles through one ring
// of shared-memory stages.  Phi does not depend on w, so its first tiles are
// already in flight while the consumers wait at the grid barrier and update
// the state: the barrier and the update hide behind the Phi stream.
//
// Every wait is bounded (psf_sm100.cuh): a wait that gives up records a code
// in the context's error word.  A consumer warp whose wait gave up stops
// waiting but keeps walking the same tiles and named barriers as the others,
// so no barrier is left short; the producer waits (bounded) for the copies it
// still has in flight before the CTA exits.
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
constexpr int STAGES = 8;
constexpr uint32_t STAGE_BYTES = 16384;  // one Phi tile; a C tile uses half a stage
constexpr int CT_ROWS = 32, CT_COLS = 64;
constexpr uint32_t CT_BYTES = CT_ROWS * CT_COLS * 4;
constexpr int RT_FACES = 64, RT_MODES = 64;
constexpr uint32_t RT_BYTES = RT_FACES * RT_MODES * 4;

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

// All CTAs (co-resident: cooperative launch) meet here; false if the wait
// gave up.  `bar` is zeroed before every launch.
__device__ __forceinline__ bool grid_barrier(unsigned int *bar, int *err)
{
    __threadfence();
    atomicAdd(bar, 1u);
    const unsigned long long t0 = globaltimer();
    for (;;) {
        unsigned int v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
        if (v >= gridDim.x) break;
        if (globaltimer() - t0 > PSF_WAIT_LIMIT_NS) {
            record_error(err, ERR_GRID_SYNC);
            return false;
        }
        __nanosleep(64);
    }
    __threadfence();
    return true;
}

// The ring position of the consumers (and of the producer).
struct Ring {
    int stage = 0;
    uint32_t phase = 0;
    __device__ __forceinline__ void next()
    {
        if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
        }
    }
};

}  // namespace

struct CoeffArgs {
    int N, KC, RC, KS;
    long long n_active;
    double *w;                  // [N] w^n in, w^{n+1} out (CTA 0)
    double *dwpart;             // [N][RC]
    const double *lam, *force;  // [N]
    StateParams sp;
    unsigned int *grid_bar;
    unsigned long long *step_ctr;
    const int32_t *faces;       // [n_active] reference face id of each Phi row
    const int32_t *pair_dst;    // [n_active][2] face-pair slots
    float *u;                   // [n_faces]
    float *pairs;               // float view of [3][V] float2
    int *err;
};

__global__ void __launch_bounds__(THREADS, 1) psf_coeff_tma(const __grid_constant__ CUtensorMap tmC,
                                                            const __grid_constant__ CUtensorMap tmP, CoeffArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const int N = a.N, KC = a.KC, RC = a.RC, KS = a.KS;
    unsigned char *stages = smem;                                         // [STAGES][16 KB]
    float *wj = reinterpret_cast<float *>(smem + STAGES * STAGE_BYTES);   // [KC * 64]  w^n, FP32
    float *wr = wj + KC * CT_COLS;                                        // [KS * 64]  w^{n+1}, FP32
    float *red2 = wr + KS * RT_MODES;                                     // [2][4][64]
    double *wd = reinterpret_cast<double *>(red2 + 2 * 4 * RT_FACES);     // [RC * 32]  w^n, FP64
    double *wn = wd + RC * CT_ROWS;                                       // [N]  Euler step, FP64
    double *red = wn + ((N + 1) & ~1);                                    // [8]
    uint64_t *full = reinterpret_cast<uint64_t *>(red + 8);
    uint64_t *empty = full + STAGES;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c_tiles = N * RC;
    const int r_tiles = (int)((a.n_active + RT_FACES - 1) / RT_FACES);
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 8);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (warp == 8) {
        // ------------------------------------------------------ TMA producer
        if (lane != 0) return;
        tma_prefetch_desc(&tmC);
        tma_prefetch_desc(&tmP);
        uint32_t last_parity[STAGES];
        bool issued[STAGES];
#pragma unroll
        for (int s = 0; s < STAGES; ++s) issued[s] = false;
        Ring q;
        bool ok = true;
        for (int pass = 0; pass < 2 && ok; ++pass) {
            const int tiles = pass == 0 ? c_tiles : r_tiles, per = pass == 0 ? KC : KS;
            for (int t = blockIdx.x; ok && t < tiles; t += gridDim.x) {
                for (int ks = 0; ks < per; ++ks) {
                    if (!mbar_wait(&empty[q.stage], q.phase ^ 1u, a.err, ERR_WAIT_EMPTY)) {
                        ok = false;
                        break;
                    }
                    unsigned char *dst = stages + (size_t)q.stage * STAGE_BYTES;
                    if (pass == 0) {
                        const int k = t / RC, rc = t - k * RC;
                        mbar_arrive_expect_tx(&full[q.stage], CT_BYTES);
                        tma_load_3d(dst, &tmC, &full[q.stage], ks * CT_COLS, rc * CT_ROWS, k);
                    } else {
                        mbar_arrive_expect_tx(&full[q.stage], RT_BYTES);
                        tma_load_3d(dst, &tmP, &full[q.stage], 0, ks * RT_MODES, t);
                    }
                    issued[q.stage] = true;
                    last_parity[q.stage] = q.phase;
                    q.next();
                }
            }
        }
        // After an error, copies may still be in flight that no one consumes:
        // wait (bounded) for them before the CTA exits.
        if (*(volatile int *)a.err != 0)
            for (int s = 0; s < STAGES; ++s)
                if (issued[s]) mbar_wait(&full[s], last_parity[s], a.err, ERR_WAIT_DRAIN);
        return;
    }

    // ---------------------------------------------------------- consumers
    for (int i = threadIdx.x; i < KC * CT_COLS; i += CONSUMERS) wj[i] = i < N ? (float)a.w[i] : 0.f;
    for (int i = threadIdx.x; i < RC * CT_ROWS; i += CONSUMERS) wd[i] = i < N ? a.w[i] : 0.0;
    consumer_bar();
    Ring q;
    bool ok = true;

    // 1. contraction.  Thread (r, cg): row r, columns cg*4..+3 and 32+cg*4..+3.
    {
        const int r = threadIdx.x >> 3, cg = threadIdx.x & 7;
        for (int t = blockIdx.x; t < c_tiles; t += gridDim.x) {
            const int k = t / RC, rc = t - k * RC;
            float part = 0.f;
            for (int ks = 0; ks < KC; ++ks) {
                if (ok && !mbar_wait(&full[q.stage], q.phase, a.err, ERR_WAIT_FULL)) ok = false;
                if (ok) {
                    const float *row = reinterpret_cast<const float *>(stages + (size_t)q.stage * STAGE_BYTES) +
                                       r * CT_COLS;
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
                if (lane == 0) mbar_arrive(&empty[q.stage]);
                q.next();
            }
            const double tot = consumer_sum(wd[rc * CT_ROWS + r] * (double)part, red);
            if (threadIdx.x == 0) a.dwpart[(size_t)k * RC + rc] = tot;
        }
    }

    // 2. grid barrier: every partial is written.
    if (threadIdx.x == 0) grid_barrier(a.grid_bar, a.err);
    consumer_bar();

    // 3. FP64 state update in the reference's order (psfsolver.cpp:37-59),
    // the same arithmetic in every CTA.
    {
        double e1 = 0.0, e2 = 0.0;
        for (int i = threadIdx.x; i < N; i += CONSUMERS) {
            const double wi = wd[i];
            double dw = 0.0;
            for (int c = 0; c < RC; ++c) dw += __ldcg(a.dwpart + (size_t)i * RC + c);
            const double w1 = wi + a.sp.dt * dw;
            wn[i] = w1;
            e1 += wi * wi;
            e2 += w1 * w1;
        }
        e1 = consumer_sum(e1, red);
        e2 = consumer_sum(e2, red);
        const double scale = (a.sp.flags & PSF_FLAG_RENORM) ? sqrt(e1 / e2) : 1.0;
        for (int i = threadIdx.x; i < KS * RT_MODES; i += CONSUMERS) {
            float f = 0.f;
            if (i < N) {
                double v = wn[i] * scale;
                v *= exp(a.sp.visc_signed * a.lam[i] * a.sp.dt);
                if (a.sp.flags & PSF_FLAG_FORCING) v += a.sp.dt * a.force[i];
                f = (float)v;
                if (blockIdx.x == 0) a.w[i] = v;
            }
            wr[i] = f;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) *a.step_ctr += 1ull;
        consumer_bar();
    }

    // 4. reconstruction.  Thread (g, f): face f of the tile, modes g*16..+15 of
    // every stage.  Threads 0..63 also write the tile's faces: their
    // destinations are loaded before the tile's stages are waited for, and the
    // partial sums go through one of two shared buffers, so a tile needs one
    // barrier and the next tile's sums start while its faces are written.
    {
        const int f = threadIdx.x & 63, g = threadIdx.x >> 6;
        int buf = 0;
        for (int t = blockIdx.x; t < r_tiles; t += gridDim.x, buf ^= 1) {
            const long long row = (long long)t * RT_FACES + threadIdx.x;
            int32_t dst = -1, d0 = -1, d1 = -1;
            if (threadIdx.x < RT_FACES && row < a.n_active) {
                dst = __ldg(a.faces + row);
                d0 = __ldg(a.pair_dst + 2 * row);
                d1 = __ldg(a.pair_dst + 2 * row + 1);
            }
            float acc = 0.f;
            for (int ks = 0; ks < KS; ++ks) {
                if (ok && !mbar_wait(&full[q.stage], q.phase, a.err, ERR_WAIT_FULL)) ok = false;
                if (ok) {
                    const float *st = reinterpret_cast<const float *>(stages + (size_t)q.stage * STAGE_BYTES) +
                                      (g * 16) * RT_FACES + f;
                    const float *wm = wr + ks * RT_MODES + g * 16;
#pragma unroll
                    for (int m = 0; m < 16; ++m) acc = fmaf(st[m * RT_FACES], wm[m], acc);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[q.stage]);
                q.next();
            }
            float *rb = red2 + buf * 4 * RT_FACES;
            rb[g * RT_FACES + f] = acc;
            consumer_bar();
            if (ok && dst >= 0) {
                const float v = (rb[threadIdx.x] + rb[RT_FACES + threadIdx.x]) +
                                (rb[2 * RT_FACES + threadIdx.x] + rb[3 * RT_FACES + threadIdx.x]);
                a.u[dst] = v;
                if (d0 >= 0) a.pairs[d0] = v;
                if (d1 >= 0) a.pairs[d1] = v;
            }
        }
    }
}

// ---------------------------------------------------------------- host
int contract_tma_row_chunks(int N) { return (N + CT_ROWS - 1) / CT_ROWS; }

int coeff_tma_smem_bytes(int N)
{
    const int KC = (N + CT_COLS - 1) / CT_COLS, RC = contract_tma_row_chunks(N), KS = (N + RT_MODES - 1) / RT_MODES;
    return STAGES * (int)STAGE_BYTES + KC * CT_COLS * 4 + KS * RT_MODES * 4 + 2 * 4 * RT_FACES * 4 +
           RC * CT_ROWS * 8 + ((N + 1) & ~1) * 8 + 8 * 8 + 2 * STAGES * 8;
}

int make_plain_tma_maps(const PlainDev &d, CUtensorMap *tmC, CUtensorMap *tmP)
{
    // C: [k][a][j] FP32, j padded to Np (a multiple of 4: 16-byte rows).
    const uint64_t dc[3] = {(uint64_t)d.Np, (uint64_t)d.N, (uint64_t)d.N};
    const uint64_t sc[2] = {(uint64_t)d.Np * 4, (uint64_t)d.N * d.Np * 4};
    const uint32_t bc[3] = {CT_COLS, CT_ROWS, 1};
    int rc = encode_tensor_map_f32(tmC, const_cast<float *>(d.C), 3, dc, sc, bc);
    if (rc != PSF_OK) return rc;
    // Phi: [tile][i][64 faces] FP32 (ldp = whole tiles); a box is 64 modes of one
    // tile, 16 KB of contiguous memory.
    const uint64_t dp[3] = {(uint64_t)RT_FACES, (uint64_t)d.N, (uint64_t)(d.ldp / RT_FACES)};
    const uint64_t sp[2] = {(uint64_t)RT_FACES * 4, (uint64_t)d.N * RT_FACES * 4};
    const uint32_t bp[3] = {RT_FACES, RT_MODES, 1};
    return encode_tensor_map_f32(tmP, const_cast<float *>(d.phiT), 3, dp, sp, bp);
}

int launch_coeff_tma(const PlainDev &d, const CUtensorMap &tmC, const CUtensorMap &tmP, int num_sms,
                     unsigned int *grid_bar, int *err, cudaStream_t st)
{
    // The dynamic shared-memory limit is a per-device attribute of the kernel;
    // it is raised once per device to what N = PSF_MAX_MODES needs.
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured & bit)) {
        e = cudaFuncSetAttribute(psf_coeff_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 coeff_tma_smem_bytes(PSF_MAX_MODES));
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        configured |= bit;
    }
    CoeffArgs a;
    a.N = d.N;
    a.KC = (d.N + CT_COLS - 1) / CT_COLS;
    a.RC = contract_tma_row_chunks(d.N);
    a.KS = (d.N + RT_MODES - 1) / RT_MODES;
    a.n_active = d.n_active;
    a.w = d.w;
    a.dwpart = d.dwpart;
    a.lam = d.lam;
    a.force = d.force;
    a.sp = d.sp;
    a.grid_bar = grid_bar;
    a.step_ctr = d.step_ctr;
    a.faces = d.faces;
    a.pair_dst = d.pair_dst;
    a.u = d.u;
    a.pairs = reinterpret_cast<float *>(d.pairs);
    a.err = err;
    // One CTA per SM (the ring takes 128 KB), all co-resident for the grid barrier.
    e = cudaMemsetAsync(grid_bar, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)std::max(1, num_sms));
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = coeff_tma_smem_bytes(d.N);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, psf_coeff_tma, tmC, tmP, a);
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_coeff_tma launch");
}

}  // namespace psf
