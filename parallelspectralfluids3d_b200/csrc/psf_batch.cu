// Batched spectral-fluid step on the 5th-generation tensor cores (sm_100a).
//
// Many instances ("slots") share one domain basis; a batch may hold several
// bases.  For the slots of one basis the two dense products of a step are
// GEMMs with the slots' coefficient vectors as the narrow operand:
//
//   contraction     Y[(k,a), b] = sum_j C[k][a][j] W[j][b]     (M = N*N, K = N)
//                   dw[k][b]    = sum_a w[a][b] Y[(k,a), b]     (epilogue, FP64)
//   reconstruction  U[f, b]     = sum_i Phi[f][i] W[i][b]       (M = F_act, K = N)
//
// C, Phi and W are stored as BF16 hi + lo pairs (x = hi + lo with both parts
// rounded to nearest) and each product is compensated:
// A_hi B_hi + A_hi B_lo + A_lo B_hi, accumulated in FP32 in TMEM.  Slots with
// fewer modes than the basis are zero-padded, which is exact: their W rows
// beyond N_b are zero, and dw_k for k >= N_b is ignored.
//
// psf_batch_step_tc is one persistent kernel over the tiles of every basis:
// warp 0 streams 128-row A tiles and the W tile through a TMA ring of
// shared-memory stages (128-byte swizzle, no multicast), warp 1 issues the
// tcgen05.mma chain for a tile into one of two TMEM accumulators, warps 2-5
// drain the other accumulator (tcgen05.ld) and run the epilogue, so loads,
// MMAs and epilogue overlap.  In the default (fused) step one cooperative
// launch runs the contraction, the FP64 state update of every slot and the
// reconstruction, separated by bounded grid barriers; the tracer
// (psf_batch_trace, the same interpolant as the single-instance path)
// completes the step.  Unfused launches (one GEMM each, plus
// psf_batch_state) serve autotuning and per-phase profiling.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "psf_b200.h"
#include "psf_batch_internal.h"
#include "psf_device.cuh"
#include "psf_internal.h"
#include "psf_sm100.cuh"

namespace psf {

using namespace sm100;

template <int BN_MAX>
struct GemmCfg {
    static constexpr int STAGES = BN_MAX == 64 ? 4 : (BN_MAX == 128 ? 3 : 2);
    static constexpr int A_BYTES = 2 * 128 * 128;  // hi + lo: 128 rows x 64 BF16
    static constexpr int B_BYTES = 2 * BN_MAX * 128;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int TMEM_COLS = 2 * BN_MAX;   // two accumulators
    static constexpr int BAR_BYTES = 256;
    static constexpr int SMEM = STAGES * STAGE_BYTES + BAR_BYTES + 1024;  // + alignment slack
};

// Work unit t of a launch: contraction units first, then reconstruction units.
// MODE 0 launches only contraction units, MODE 1 only reconstruction units,
// MODE 2 (fused) both, so the unit kind is known at compile time except there.
template <int MODE>
__device__ __forceinline__ const GemmGroup &unit_group(const StepArgs &a, int t, bool &recon, int *local)
{
    recon = MODE == 1 ? true : (MODE == 0 ? false : t >= a.c_tiles);
    int base = recon ? a.n_groups : 0;
    int u = recon ? t - a.c_tiles : t;
    int g = 0;
    while (g + 1 < a.n_groups && u >= a.g[base + g].tiles) {
        u -= a.g[base + g].tiles;
        ++g;
    }
    *local = u;
    return a.g[base + g];
}

// Work unit -> (outer index, row tile, K range [kc0, kc1)).
struct Unit {
    int outer, inner, ks, kc0, kc1;
};

__device__ __forceinline__ Unit decode_unit(const GemmGroup &G, int lt)
{
    Unit u;
    const int per_outer = G.m_inner * G.ksplit;
    u.outer = lt / per_outer;
    const int rem = lt - u.outer * per_outer;
    u.inner = rem / G.ksplit;
    u.ks = rem - u.inner * G.ksplit;
    u.kc0 = u.ks * G.kc_per;
    u.kc1 = min(G.k_chunks, u.kc0 + G.kc_per);
    return u;
}

// 32 values per lane -> lane l holds the sum over the warp of value l.
__device__ __forceinline__ float warp_reduce_scatter32f(float (&v)[32], int lane)
{
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool upper = (lane & s) != 0;
#pragma unroll
        for (int i = 0; i < s; ++i) {
            const float send = upper ? v[i] : v[i + s];
            const float keep = upper ? v[i + s] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
        }
    }
    return v[0];
}

__device__ __forceinline__ double warp_allsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void epilogue_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Grid-wide barrier of a cooperative launch: arrive, then wait (bounded) until
// `target` arrivals were counted.  Called by one thread per CTA after a CTA
// barrier, as the cooperative-groups grid sync does.
__device__ __forceinline__ bool grid_sync(unsigned int *bar, unsigned int target, int *err)
{
    __threadfence();
    atomicAdd(bar, 1u);
    const unsigned long long t0 = globaltimer();
    for (;;) {
        unsigned int v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
        if (v >= target) break;
        if (globaltimer() - t0 > PSF_WAIT_LIMIT_NS) {
            record_error(err, ERR_GRID_SYNC);
            return false;
        }
        __nanosleep(64);
    }
    __threadfence();
    return true;
}

__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 *hi, __nv_bfloat16 *lo)
{
    const __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    *hi = h;
    *lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
}

// FP64 update of one slot by the 128 epilogue threads of a CTA, in the
// reference's order (psfsolver.cpp:37-59), then the new state's FP32 copy and
// BF16 hi/lo split.  Energy sums: per warp (shuffles), then the 4 warps in
// fixed order, so the result does not depend on timing.
__device__ void state_update_cta(const GroupDev *__restrict__ groups, SlotDev &s, int et, double *red)
{
    const int lane = et & 31, ew = et >> 5;
    if (!s.active) return;  // uniform over the 128 threads
    if (s.target != 0ull && s.step >= s.target) {
        if (et == 0) s.stepped = 0;
        return;
    }
    const GroupDev &G = groups[s.group];
    const int b = s.slot, N = s.n_modes, parts = G.nparts;
    double *w = G.w + (size_t)b * G.N;
    double e1 = 0.0, e2 = 0.0;
    for (int i = et; i < N; i += 128) {
        double dw = 0.0;
        const double *dp = G.dwpart + (size_t)i * parts * G.cap + b;
        for (int p = 0; p < parts; ++p) dw += dp[(size_t)p * G.cap];
        const double wi = w[i];
        const double w1 = wi + s.dt * dw;
        w[i] = w1;
        e1 += wi * wi;
        e2 += w1 * w1;
    }
    e1 = warp_allsum(e1);
    e2 = warp_allsum(e2);
    if (lane == 0) {
        red[ew] = e1;
        red[4 + ew] = e2;
    }
    epilogue_bar();
    e1 = red[0] + red[1] + red[2] + red[3];
    e2 = red[4] + red[5] + red[6] + red[7];
    const double scale = (s.flags & PSF_FLAG_RENORM) ? sqrt(e1 / e2) : 1.0;
    __nv_bfloat16 *Whi = reinterpret_cast<__nv_bfloat16 *>(G.W) + (size_t)b * G.Nj;
    __nv_bfloat16 *Wlo = Whi + (size_t)G.bn * G.Nj;
    for (int i = et; i < N; i += 128) {
        double v = w[i] * scale;
        v *= exp(s.visc_signed * G.lam[i] * s.dt);
        if (s.flags & PSF_FLAG_FORCING) v += s.dt * G.force[(size_t)b * G.N + i];
        w[i] = v;
        G.wf[(size_t)b * G.N + i] = (float)v;
        split_bf16(v, Whi + i, Wlo + i);
    }
    epilogue_bar();  // red[] is reused by the next slot
    if (et == 0) {
        s.step += 1ull;
        s.stepped = 1;
    }
}

// One launch of the tensor-core step.  Warp 0: TMA producer; warp 1: MMA
// issuer; warps 2-5: TMEM epilogue.  Unfused launches run their contraction
// or reconstruction units.  A fused launch (cooperative) is one whole step of
// the coefficient pipeline: the epilogue warps first update every slot's
// state from the contraction partials of the previous launch (FP64, one CTA
// per slot), a grid barrier makes the new coefficients visible, and then
// one sweep runs the reconstruction of the new state together with the
// contraction that the next step's update will use (both need only the new
// coefficients).  During the update the producer already loads the first
// tiles of C and Phi, which do not depend on the state, and issues their
// coefficient (W) loads once the barrier has passed.
template <int BN_MAX, int MODE>
__global__ void __launch_bounds__(GEMM_THREADS, 1) psf_batch_step_tc(const __grid_constant__ StepArgs args)
{
    using Cfg = GemmCfg<BN_MAX>;
    constexpr int STAGES = Cfg::STAGES;
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw_addr = smem_u32(smem_raw);
    unsigned char *smem = smem_raw + ((1024u - (raw_addr & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + STAGES * Cfg::STAGE_BYTES);
    uint64_t *full = bars;
    uint64_t *empty = bars + STAGES;
    uint64_t *acc_full = bars + 2 * STAGES;
    uint64_t *acc_empty = acc_full + 2;
    uint64_t *wready = acc_empty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(wready + 1);
    double *red = reinterpret_cast<double *>(wready + 2);  // 8 doubles (bytes 8*(2*STAGES+6) .. +64)

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *err = args.err;
    const int total = args.c_tiles + args.r_tiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 128);
        }
        mbar_init(wready, 1);
        mbar_fence_init();
        for (int g = 0; g < 2 * args.n_groups; ++g) {
            tma_prefetch_desc(&args.g[g].tmA);
            tma_prefetch_desc(&args.g[g].tmB);
        }
    }
    if (warp == 1) tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------------------------------------------- TMA producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t last_parity[STAGES];
            bool issued[STAGES];
            for (int s = 0; s < STAGES; ++s) issued[s] = false;
            // Reconstruction stages whose W load waits for the state update.
            int pend_stage[STAGES], pend_kc[STAGES], pend_t[STAGES];
            int npend = 0;
            bool w_ok = MODE != 2;
            bool ok = true;
            auto flush = [&]() -> bool {
                if (!mbar_wait(wready, 0u, err, ERR_WAIT_STATE)) return false;
                for (int i = 0; i < npend; ++i) {
                    bool rc;
                    int lt;
                    const GemmGroup &G = unit_group<MODE>(args, pend_t[i], rc, &lt);
                    unsigned char *sB = smem + pend_stage[i] * Cfg::STAGE_BYTES + Cfg::A_BYTES;
                    tma_load_3d(sB, &G.tmB, &full[pend_stage[i]], pend_kc[i] * 64, 0, 0);
                }
                npend = 0;
                w_ok = true;
                return true;
            };
            for (int t = blockIdx.x; ok && t < total; t += gridDim.x) {
                bool recon;
                int lt;
                const GemmGroup &G = unit_group<MODE>(args, t, recon, &lt);
                const Unit un = decode_unit(G, lt);
                for (int kc = un.kc0; kc < un.kc1; ++kc) {
                    if (!mbar_wait(&empty[stage], phase ^ 1u, err, ERR_WAIT_EMPTY)) {
                        ok = false;
                        break;
                    }
                    unsigned char *sA = smem + stage * Cfg::STAGE_BYTES;
                    unsigned char *sB = sA + Cfg::A_BYTES;
                    mbar_arrive_expect_tx(&full[stage], G.tx_bytes);
                    tma_load_4d(sA, &G.tmA, &full[stage], kc * 64, un.inner * 128, 0, un.outer);
                    if (!w_ok) {
                        pend_stage[npend] = stage;
                        pend_kc[npend] = kc;
                        pend_t[npend] = t;
                        ++npend;
                    } else {
                        tma_load_3d(sB, &G.tmB, &full[stage], kc * 64, 0, 0);
                    }
                    issued[stage] = true;
                    last_parity[stage] = phase;
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                    if (npend == STAGES && !flush()) {
                        ok = false;
                        break;
                    }
                }
            }
            if (ok && npend > 0) ok = flush();
            // After an error, copies may still be in flight that no one
            // consumes: wait (bounded) for them before the CTA exits.
            if (*(volatile int *)err != 0)
                for (int s = 0; s < STAGES; ++s)
                    if (issued[s]) mbar_wait(&full[s], last_parity[s], err, ERR_WAIT_DRAIN);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int abuf = 0;
            uint32_t aphase = 0;
            bool ok = true;
            for (int t = blockIdx.x; ok && t < total; t += gridDim.x) {
                bool recon;
                int lt;
                const GemmGroup &G = unit_group<MODE>(args, t, recon, &lt);
                const Unit un = decode_unit(G, lt);
                if (!mbar_wait(&acc_empty[abuf], aphase ^ 1u, err, ERR_WAIT_ACC_EMPTY)) break;
                tc_fence_after();
                const uint32_t d = tmem_base + (uint32_t)(abuf * BN_MAX);
                const uint32_t idesc = idesc_bf16_f32(128, G.bn);
                for (int kc = un.kc0; kc < un.kc1; ++kc) {
                    if (!mbar_wait(&full[stage], phase, err, ERR_WAIT_FULL)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(smem + stage * Cfg::STAGE_BYTES);
                    const uint32_t b0 = a0 + Cfg::A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const uint64_t ah = desc_kmajor_sw128(a0 + kk * 32);
                        const uint64_t al = desc_kmajor_sw128(a0 + 128 * 128 + kk * 32);
                        const uint64_t bh = desc_kmajor_sw128(b0 + kk * 32);
                        const uint64_t bl = desc_kmajor_sw128(b0 + (uint32_t)G.bn * 128u + kk * 32);
                        mma_bf16(d, ah, bh, idesc, (kc != un.kc0 || kk != 0) ? 1u : 0u);
                        mma_bf16(d, ah, bl, idesc, 1u);
                        mma_bf16(d, al, bh, idesc, 1u);
                    }
                    mma_commit(&empty[stage]);
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                mma_commit(&acc_full[abuf]);
                if (++abuf == 2) {
                    abuf = 0;
                    aphase ^= 1u;
                }
            }
        }
    } else {
        // -------------------------------------------------------- epilogue
        const int q = warp & 3;   // TMEM lanes 32q .. 32q+31 belong to this warp
        const int row = q * 32 + lane;
        int abuf = 0;
        uint32_t aphase = 0;
        if (MODE == 2) {
            // Every slot's state update (one CTA per slot), then a grid
            // barrier before any coefficient (W) load of the sweep.
            const int et = threadIdx.x - 64;
            for (int s = blockIdx.x; s < args.n_slots; s += gridDim.x)
                state_update_cta(args.groups, args.slots[s], et, red);
            // The new coefficients are read next by TMA (the async proxy).
            asm volatile("fence.proxy.async.global;" ::: "memory");
            epilogue_bar();
            if (threadIdx.x == 64) {
                if (grid_sync(args.grid_bar, gridDim.x, err)) mbar_arrive(wready);
            }
            epilogue_bar();
            // The epilogue reads other CTAs' new state (wf) below with
            // ordinary (L1-cached) loads: order them after the barrier.
            __threadfence();
        }
        for (int t = blockIdx.x; t < total; t += gridDim.x) {
            bool recon;
            int lt;
            const GemmGroup &G = unit_group<MODE>(args, t, recon, &lt);
            const Unit un = decode_unit(G, lt);
            const int outer = un.outer, inner = un.inner;
            // Contraction: the state values of this warp's rows for the first
            // slots are loaded while the accumulator is still being computed.
            // With at most 64 MMA columns both 32-slot chunks are loaded up
            // front; with more, each later chunk is loaded one chunk ahead of
            // its use (two ahead measured 22 % slower at 256 columns).
            constexpr bool kTwoAhead = BN_MAX <= 64;
            float wa[32], wb[32];
            const int a_row = inner * 128 + row;
            const bool arow = !recon && a_row < G.n_rows;
            auto load_w = [&](float(&dst)[32], int c0) {
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int b = c0 + c;
                    dst[c] = (arow && b < G.cap) ? G.wf[(size_t)b * G.ldw + a_row] : 0.f;
                }
            };
            if (!recon) {
                load_w(wa, 0);
                if (kTwoAhead && 32 < G.bn) load_w(wb, 32);
            }
            bool ok = mbar_wait(&acc_full[abuf], aphase, err, ERR_WAIT_ACC_FULL);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            tc_fence_after();
            const uint32_t tbase = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(abuf * BN_MAX);
            if (!recon) {
                // dw partial of mode k = outer over this warp's 32 rows a:
                // sum_a w[a][b] Y[a][b] for every slot b, in FP32.
                auto chunk = [&](int c0, float(&wv)[32]) {
                    float y[32];
                    tmem_ld32(tbase + (uint32_t)c0, y);
#pragma unroll
                    for (int c = 0; c < 32; ++c) y[c] *= wv[c];
                    if (kTwoAhead) {
                        if (c0 + 64 < G.bn) load_w(wv, c0 + 64);
                    } else if (c0 + 32 < G.bn) {
                        load_w(wv, c0 + 32);
                    }
                    const float s = warp_reduce_scatter32f(y, lane);
                    const int b = c0 + lane;
                    if (b < G.cap)
                        G.dwpart[((size_t)outer * G.nparts + (inner * G.ksplit + un.ks) * 4 + q) * G.cap + b] =
                            (double)s;
                };
                if (kTwoAhead) {
                    for (int c0 = 0; c0 < G.bn; c0 += 64) {
                        chunk(c0, wa);
                        if (c0 + 32 < G.bn) chunk(c0 + 32, wb);
                    }
                } else {
                    for (int c0 = 0; c0 < G.bn; c0 += 32) chunk(c0, wa);
                }
            } else {
                // Face velocities of this warp's 32 rows, scattered into the
                // per-voxel face pairs (each face lands in its two voxels) of
                // every slot that stepped: the tracer reads no others, so an
                // empty or finished slot costs no stores.
                const long long f = (long long)inner * 128 + row;
                const bool frow = f < G.n_rows;
                const int32_t d0 = frow ? __ldg(G.pair_dst + 2 * f) : -1;
                const int32_t d1 = frow ? __ldg(G.pair_dst + 2 * f + 1) : -1;
                for (int c0 = 0; c0 < G.bn; c0 += 32) {
                    const int bl = c0 + lane;
                    const unsigned stepped =
                        __ballot_sync(0xffffffffu, bl < G.cap && G.slot_of[bl].stepped != 0);
                    float y[32];
                    tmem_ld32(tbase + (uint32_t)c0, y);
                    if (frow && stepped) {
#pragma unroll
                        for (int c = 0; c < 32; ++c) {
                            const int b = c0 + c;
                            if ((stepped >> c) & 1u) {
                                float *pr = G.pairs + (size_t)b * G.pair_floats;
                                if (d0 >= 0) pr[d0] = y[c];
                                if (d1 >= 0) pr[d1] = y[c];
                            }
                        }
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&acc_empty[abuf]);
            if (++abuf == 2) {
                abuf = 0;
                aphase ^= 1u;
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, Cfg::TMEM_COLS);
    }
}

// ------------------------------------------------------------ state update
// FP64 update of one slot in the reference's order (psfsolver.cpp:37-59),
// then the new state's BF16 hi/lo split for the next products.
__global__ void __launch_bounds__(256) psf_batch_state(const GroupDev *__restrict__ groups,
                                                       SlotDev *__restrict__ slots)
{
    __shared__ double red[8];
    __shared__ double wnew[PSF_MAX_MODES];
    SlotDev &s = slots[blockIdx.x];
    if (!s.active) return;
    if (s.target != 0ull && s.step >= s.target) {
        if (threadIdx.x == 0) s.stepped = 0;
        return;
    }
    const GroupDev &G = groups[s.group];
    const int b = s.slot, N = s.n_modes, parts = G.nparts;
    double *w = G.w + (size_t)b * G.N;
    double e1 = 0.0, e2 = 0.0;
    for (int i = threadIdx.x; i < N; i += 256) {
        double dw = 0.0;
        const double *dp = G.dwpart + (size_t)i * parts * G.cap + b;
        for (int p = 0; p < parts; ++p) dw += dp[(size_t)p * G.cap];
        const double wi = w[i];
        const double w1 = wi + s.dt * dw;
        wnew[i] = w1;
        e1 += wi * wi;
        e2 += w1 * w1;
    }
    e1 = block_sum_256(e1, red);
    e2 = block_sum_256(e2, red);
    const double scale = (s.flags & PSF_FLAG_RENORM) ? sqrt(e1 / e2) : 1.0;
    __nv_bfloat16 *Whi = reinterpret_cast<__nv_bfloat16 *>(G.W) + (size_t)b * G.Nj;
    __nv_bfloat16 *Wlo = Whi + (size_t)G.bn * G.Nj;
    for (int i = threadIdx.x; i < N; i += 256) {
        double v = wnew[i] * scale;
        v *= exp(s.visc_signed * G.lam[i] * s.dt);
        if (s.flags & PSF_FLAG_FORCING) v += s.dt * G.force[(size_t)b * G.N + i];
        w[i] = v;
        G.wf[(size_t)b * G.N + i] = (float)v;
        split_bf16(v, Whi + i, Wlo + i);
    }
    if (threadIdx.x == 0) {
        s.step += 1ull;
        s.stepped = 1;
    }
}

// BF16 split of one slot's current state (after it was set from the host).
__global__ void psf_batch_pack(const GroupDev *__restrict__ groups, const SlotDev *__restrict__ slots, int sg)
{
    const SlotDev &s = slots[sg];
    const GroupDev &G = groups[s.group];
    __nv_bfloat16 *Whi = reinterpret_cast<__nv_bfloat16 *>(G.W) + (size_t)s.slot * G.Nj;
    __nv_bfloat16 *Wlo = Whi + (size_t)G.bn * G.Nj;
    for (int i = threadIdx.x; i < G.Nj; i += blockDim.x) {
        const double v = (s.active && i < s.n_modes) ? G.w[(size_t)s.slot * G.N + i] : 0.0;
        split_bf16(v, Whi + i, Wlo + i);
        if (i < G.N) G.wf[(size_t)s.slot * G.N + i] = (float)v;
    }
}

// ------------------------------------------------------------------ tracer
// Every occupied slot's particles form one index space through the prefix
// sums of the slots' particle counts; a particle finds its slot by binary
// search in shared memory.  Slots that did not advance this step (step limit
// reached) are skipped.
__global__ void __launch_bounds__(128, 5) psf_batch_trace(const GroupDev *__restrict__ groups,
                                                          const SlotDev *__restrict__ slots,
                                                          const long long *__restrict__ prefix, int n_slots)
{
    __shared__ long long pre[BATCH_MAX_ALL_SLOTS + 1];
    for (int i = threadIdx.x; i <= n_slots; i += blockDim.x) pre[i] = prefix[i];
    __syncthreads();
    const long long total = pre[n_slots];
    const long long stride = (long long)gridDim.x * blockDim.x;
    // Parameters of the slot the thread is in, reloaded only when it changes.
    int cur = -1;
    bool live = false;
    size_t base = 0;
    TraceParams tp;
    uint64_t step = 0;
    const float2 *pairs = nullptr;
    const GroupDev *G = nullptr;
    for (long long gi = (long long)blockIdx.x * blockDim.x + threadIdx.x; gi < total; gi += stride) {
        if (cur < 0 || gi >= pre[cur + 1]) {
            int lo = cur < 0 ? 0 : cur;
            int walk = 0;
            while (pre[lo + 1] <= gi && walk < 8) {
                ++lo;
                ++walk;
            }
            if (pre[lo + 1] <= gi) {  // far away: binary search, pre[lo] <= gi < pre[hi]
                int hi = n_slots;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (pre[mid] <= gi)
                        lo = mid;
                    else
                        hi = mid;
                }
            }
            cur = lo;
            const SlotDev &s = slots[cur];
            live = s.stepped != 0;
            G = groups + s.group;
            base = (size_t)s.poff - (size_t)pre[cur];
            tp.dt = (float)s.dt;
            tp.lifetime = s.lifetime;
            tp.rk4 = s.rk4;
            tp.seed = s.seed;
            step = s.step - 1ull;
            pairs = G->pairs + (size_t)s.slot * 3 * (size_t)G->V;
        }
        if (!live) continue;
        const size_t idx = base + (size_t)gi;
        float4 p = G->parts[idx];
        p = advance_particle(p, G->grid, pairs, tp, step, G->perm, idx);
        G->parts[idx] = p;
    }
}

// --------------------------------------------------------------- launchers
int batch_gemm_smem_bytes(int bn_max)
{
    switch (bn_max) {
    case 64: return GemmCfg<64>::SMEM;
    case 128: return GemmCfg<128>::SMEM;
    case 256: return GemmCfg<256>::SMEM;
    default: return -1;
    }
}

template <int BN, int MODE>
static int launch_tc_t(const StepArgs &args, int grid, cudaStream_t st)
{
    // The shared-memory limit is a per-device attribute of the kernel.
    static unsigned long long configured = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured & bit)) {
        e = cudaFuncSetAttribute(psf_batch_step_tc<BN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 GemmCfg<BN>::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(psf_batch_step_tc)");
        configured |= bit;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(GEMM_THREADS);
    cfg.dynamicSmemBytes = GemmCfg<BN>::SMEM;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = MODE == 2 ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, psf_batch_step_tc<BN, MODE>, args);
    if (e != cudaSuccess) return cuda_fail(e, "psf_batch_step_tc launch");
    return PSF_OK;
}

template <int MODE>
static int launch_tc_mode(const StepArgs &args, int bn_max, int grid, cudaStream_t st)
{
    switch (bn_max) {
    case 64: return launch_tc_t<64, MODE>(args, grid, st);
    case 128: return launch_tc_t<128, MODE>(args, grid, st);
    case 256: return launch_tc_t<256, MODE>(args, grid, st);
    }
    return fail(PSF_ERR_UNSUPPORTED, "GEMM variant must have 64, 128 or 256 columns");
}

int launch_batch_step_tc(const StepArgs &args, int bn_max, int grid, cudaStream_t st)
{
    const int total = args.c_tiles + args.r_tiles;
    if (total <= 0 && !args.fused) return PSF_OK;
    if (!args.fused) grid = std::min(grid, total);
    grid = std::max(1, grid);
    for (int g = 0; g < 2 * args.n_groups; ++g) {
        const bool used = g < args.n_groups ? args.c_tiles > 0 : args.r_tiles > 0;
        if (used && (args.g[g].bn > bn_max || args.g[g].bn % 16 != 0 || args.g[g].bn < 16))
            return fail(PSF_ERR_INVALID, "GEMM group N tile does not fit the kernel variant");
    }
    if (args.fused) return launch_tc_mode<2>(args, bn_max, grid, st);
    if (args.r_tiles == 0) return launch_tc_mode<0>(args, bn_max, grid, st);
    if (args.c_tiles == 0) return launch_tc_mode<1>(args, bn_max, grid, st);
    return fail(PSF_ERR_INVALID, "an unfused launch runs either contraction or reconstruction units");
}

// Largest persistent grid a cooperative launch of the variant can hold.
int max_fused_grid(int bn_max, int num_sms)
{
    int per_sm = 0;
    cudaError_t e = cudaSuccess;
    switch (bn_max) {
    case 64:
        cudaFuncSetAttribute(psf_batch_step_tc<64, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmCfg<64>::SMEM);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psf_batch_step_tc<64, 2>, GEMM_THREADS,
                                                          GemmCfg<64>::SMEM);
        break;
    case 128:
        cudaFuncSetAttribute(psf_batch_step_tc<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             GemmCfg<128>::SMEM);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psf_batch_step_tc<128, 2>, GEMM_THREADS,
                                                          GemmCfg<128>::SMEM);
        break;
    default:
        cudaFuncSetAttribute(psf_batch_step_tc<256, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             GemmCfg<256>::SMEM);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psf_batch_step_tc<256, 2>, GEMM_THREADS,
                                                          GemmCfg<256>::SMEM);
        break;
    }
    if (e != cudaSuccess) return 0;
    return per_sm * num_sms;
}

int launch_batch_state(const GroupDev *groups, SlotDev *slots, int n_slots, cudaStream_t st)
{
    if (n_slots <= 0) return PSF_OK;
    psf_batch_state<<<n_slots, 256, 0, st>>>(groups, slots);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_batch_state launch");
}

int launch_batch_pack(const GroupDev *groups, const SlotDev *slots, int slot_global, cudaStream_t st)
{
    psf_batch_pack<<<1, 256, 0, st>>>(groups, slots, slot_global);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_batch_pack launch");
}

int batch_trace_grid(int num_sms)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psf_batch_trace, 128, 0) != cudaSuccess || per_sm < 1)
        per_sm = 4;
    return num_sms * per_sm;
}

int launch_batch_trace(const GroupDev *groups, const SlotDev *slots, const long long *prefix, int n_slots, int grid,
                       cudaStream_t st)
{
    if (n_slots < 1 || n_slots > BATCH_MAX_ALL_SLOTS) return fail(PSF_ERR_INVALID, "slot count out of range");
    psf_batch_trace<<<grid, 128, 0, st>>>(groups, slots, prefix, n_slots);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_batch_trace launch");
}

// ------------------------------------------------------------ host helpers
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_tensor_map(CUtensorMap *map, void *base, int rank, const uint64_t *dims, const uint64_t *strides_bytes,
                      const uint32_t *box)
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
            return fail(PSF_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    cuuint64_t d[5];
    cuuint64_t s[4];
    cuuint32_t bx[5], es[5];
    for (int i = 0; i < rank; ++i) {
        d[i] = dims[i];
        bx[i] = box[i];
        es[i] = 1;
        if (i + 1 < rank) s[i] = strides_bytes[i];
    }
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, base, d, s, bx, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(PSF_ERR_CUDA, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
    return PSF_OK;
}

void split_bf16_host(double x, uint16_t *hi, uint16_t *lo)
{
    const __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    const __nv_bfloat16 l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
    std::memcpy(hi, &h, 2);
    std::memcpy(lo, &l, 2);
}

}  // namespace psf
