// B200 (sm_100a) spectral-fluid step engine: kernels and the C ABI of
// include/psf_b200.h for single-instance contexts.
//
// One step (the reference's PSFSolver::integrate, Solver/SolverImpl/
// psfsolver.cpp:21-234) is three kernels, captured once into a CUDA graph:
//
//   1. psf_contract_state  dw_k = sum_a w_a sum_j C[k][a][j] w_j over an FP32
//      C streamed with 128-bit loads, FP64 accumulation; the last CTA to
//      finish (atomic ticket, no spinning) applies the FP64 state update:
//      Euler step, energy renormalisation, viscous decay, forcing.
//      (replaces simulation.cl:207-311 and :356-394, five OpenCL kernels)
//   2. psf_reconstruct     u = Phi w with Phi stored as contiguous 64-face
//      tiles (the tracer's face signs folded in); scatter to the reference
//      face numbering and to the per-voxel face pairs.
//      (replaces simulation.cl:313-354)
//   3. psf_trace           one thread per particle, trilinear staggered
//      interpolation from the signed face field, RK1 or RK4, box clamp,
//      lifetime and respawn.  (replaces simulation.cl:33-205)
//
// This file also holds the particle ordering kernels and the error helpers.

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "psf_b200.h"
#include "psf_internal.h"
#include "psf_device.cuh"

namespace psf {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(e == cudaErrorMemoryAllocation ? PSF_ERR_NOMEM : PSF_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

// --------------------------------------------- programmatic dependent launch
// The three step kernels run back to back in one stream.  Each one loads only
// constant data (C rows, Phi tiles, face maps) before griddepcontrol.wait, and
// lets its own dependents launch only after that wait: at most two kernels
// are in flight, and the second never reads what the first is still writing.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// ------------------------------------------------------- 1. contraction
// Block b handles mode k = b / S and row slice s = b % S of C_k.  Lane l of a
// warp owns columns [4l + 128c, 4l + 128c + 4) for c < CH; warps walk rows a.
// Each lane accumulates sum_a w_a * (C[k][a][j..j+3] . w[j..j+3]) in FP64, so
// no per-row reduction is needed; one block reduction at the end.  The first
// PF rows of every warp are loaded before the grid-dependency wait (C is
// constant); the rest stream U rows per batch with w staged in shared memory.
template <int CH>
__global__ void __launch_bounds__(256) psf_contract_state(const float *__restrict__ C, int N, int Np, int S,
                                                          const double *w, double *w_next,
                                                          double *__restrict__ dwpart,
                                                          const double *__restrict__ lam,
                                                          const double *__restrict__ force, StateParams sp,
                                                          unsigned int *__restrict__ ticket,
                                                          const unsigned long long *step_ctr,
                                                          unsigned long long *step_ctr_next)
{
    constexpr int PF = CH <= 2 ? 4 : 2;
    constexpr int U = CH <= 2 ? 4 : 2;
    __shared__ double red[8];
    __shared__ int is_last;
    __shared__ double wsh[PSF_MAX_MODES];
    __shared__ double wnew[PSF_MAX_MODES];

    const int k = blockIdx.x / S;
    const int s = blockIdx.x - k * S;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rows = (N + S - 1) / S;
    const int a0 = s * rows;
    const int a1 = min(N, a0 + rows);
    const float *Ck = C + (size_t)k * N * Np;

    float4 pre[PF][CH];
#pragma unroll
    for (int r = 0; r < PF; ++r) {
        const int a = a0 + warp + 8 * r;
        const float4 *row = reinterpret_cast<const float4 *>(Ck + (size_t)a * Np);
#pragma unroll
        for (int c = 0; c < CH; ++c)
            pre[r][c] = (a < a1 && c * 128 + lane * 4 < Np) ? __ldg(row + c * 32 + lane)
                                                            : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    grid_dependency_wait();
    launch_dependents();
    for (int i = threadIdx.x; i < N; i += 256) wsh[i] = w[i];
    __syncthreads();

    float wj[CH][4];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int col = c * 128 + lane * 4 + q;
            wj[c][q] = col < N ? (float)wsh[col] : 0.f;
        }
    }
    double acc = 0.0;
#pragma unroll
    for (int r = 0; r < PF; ++r) {
        const int a = a0 + warp + 8 * r;
        if (a < a1) {
            float part = 0.f;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                part = fmaf(pre[r][c].x, wj[c][0], part);
                part = fmaf(pre[r][c].y, wj[c][1], part);
                part = fmaf(pre[r][c].z, wj[c][2], part);
                part = fmaf(pre[r][c].w, wj[c][3], part);
            }
            acc = fma(wsh[a], (double)part, acc);
        }
    }
    for (int ab = a0 + warp + 8 * PF; ab < a1; ab += 8 * U) {
        float4 v[U][CH];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int a = ab + 8 * u;
            const float4 *row = reinterpret_cast<const float4 *>(Ck + (size_t)a * Np);
#pragma unroll
            for (int c = 0; c < CH; ++c)
                v[u][c] = (a < a1 && c * 128 + lane * 4 < Np) ? __ldg(row + c * 32 + lane)
                                                              : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int a = ab + 8 * u;
            if (a < a1) {
                float part = 0.f;
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    part = fmaf(v[u][c].x, wj[c][0], part);
                    part = fmaf(v[u][c].y, wj[c][1], part);
                    part = fmaf(v[u][c].z, wj[c][2], part);
                    part = fmaf(v[u][c].w, wj[c][3], part);
                }
                acc = fma(wsh[a], (double)part, acc);
            }
        }
    }
    const double tot = block_sum_256(acc, red);
    if (threadIdx.x == 0) {
        dwpart[blockIdx.x] = tot;
        __threadfence();
        const unsigned int prev = atomicAdd(ticket, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();

    // Last block: FP64 state update in the reference's order
    // (psfsolver.cpp:37-59).
    double e1 = 0.0, e2 = 0.0;
    for (int i = threadIdx.x; i < N; i += 256) {
        const double wi = wsh[i];
        double dw = 0.0;
        for (int q = 0; q < S; ++q) dw += __ldcg(dwpart + i * S + q);
        const double w1 = wi + sp.dt * dw;
        wnew[i] = w1;
        e1 += wi * wi;
        e2 += w1 * w1;
    }
    e1 = block_sum_256(e1, red);
    e2 = block_sum_256(e2, red);
    const double scale = (sp.flags & PSF_FLAG_RENORM) ? sqrt(e1 / e2) : 1.0;
    for (int i = threadIdx.x; i < N; i += 256) {
        double v = wnew[i] * scale;
        v *= exp(sp.visc_signed * lam[i] * sp.dt);
        if (sp.flags & PSF_FLAG_FORCING) v += sp.dt * force[i];
        w_next[i] = v;
    }
    if (threadIdx.x == 0) {
        *ticket = 0u;
        const unsigned long long n = *step_ctr;
        *step_ctr_next = n + 1ull;
    }
}


// ------------------------------------------------------ reconstruction
// 256 threads = 8 warps x 32 lanes; a block covers 128 consecutive active
// faces (4 per lane, one float4 per mode); warp g sums modes i = g (mod 8).
// Phi is stored as 64-face tiles, each mode-major ([tile][i][64]), so the
// block's two tiles are 2 x N x 256 contiguous bytes: lanes 0-15 stream one
// tile, lanes 16-31 the other.
__global__ void __launch_bounds__(256) psf_reconstruct(const float *__restrict__ phiT, long long ldp,
                                                       const int32_t *__restrict__ faces, long long n_active,
                                                       int N, const double *__restrict__ w, float *__restrict__ u,
                                                       float *__restrict__ pairs,
                                                       const int32_t *__restrict__ pair_dst)
{
    __shared__ float wsm[PSF_MAX_MODES];
    __shared__ float4 red[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long f0 = (long long)blockIdx.x * 128 + lane * 4;
    // Loads that depend on nothing go first, before w is staged: the first
    // PRE modes of this warp's share of Phi and, in warp 0, the destinations
    // of its four faces.  (Measured on the 32^3 + sphere, N = 128 workload:
    // 13.5 us against 15.3 us with the loads after the barrier.)
    constexpr int PRE = 8;
    const bool live = f0 < ldp;
    const float *base = phiT + (size_t)(f0 >> 6) * N * 64 + (f0 & 63);
    float4 v[PRE];
#pragma unroll
    for (int k = 0; k < PRE; ++k) {
        const int i = warp + 8 * k;
        v[k] = (live && i < N) ? __ldcs(reinterpret_cast<const float4 *>(base + (size_t)i * 64))
                               : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    int32_t dst[4] = {-1, -1, -1, -1}, d0[4] = {-1, -1, -1, -1}, d1[4] = {-1, -1, -1, -1};
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const long long r = f0 + q;
            if (r < n_active) {
                dst[q] = __ldg(faces + r);
                d0[q] = __ldg(pair_dst + 2 * r);
                d1[q] = __ldg(pair_dst + 2 * r + 1);
            }
        }
    }
    grid_dependency_wait();
    launch_dependents();
    for (int i = threadIdx.x; i < N; i += 256) wsm[i] = (float)w[i];
    __syncthreads();
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < PRE; ++k) {
        const int i = warp + 8 * k;
        const float wi = i < N ? wsm[i] : 0.f;
        acc.x = fmaf(v[k].x, wi, acc.x);
        acc.y = fmaf(v[k].y, wi, acc.y);
        acc.z = fmaf(v[k].z, wi, acc.z);
        acc.w = fmaf(v[k].w, wi, acc.w);
    }
    if (live) {
#pragma unroll 8
        for (int i = warp + 8 * PRE; i < N; i += 8) {
            const float4 x = __ldcs(reinterpret_cast<const float4 *>(base + (size_t)i * 64));
            const float wi = wsm[i];
            acc.x = fmaf(x.x, wi, acc.x);
            acc.y = fmaf(x.y, wi, acc.y);
            acc.z = fmaf(x.z, wi, acc.z);
            acc.w = fmaf(x.w, wi, acc.w);
        }
    }
    red[warp][lane] = acc;
    __syncthreads();
    if (warp == 0) {
        float4 t = red[0][lane];
#pragma unroll
        for (int g = 1; g < 8; ++g) {
            const float4 r = red[g][lane];
            t.x += r.x;
            t.y += r.y;
            t.z += r.z;
            t.w += r.w;
        }
        const float vals[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (dst[q] >= 0) {
                u[dst[q]] = vals[q];
                if (d0[q] >= 0) pairs[d0[q]] = vals[q];
                if (d1[q] >= 0) pairs[d1[q]] = vals[q];
            }
        }
    }
}

// Persistent grid (a whole number of resident blocks per SM) striding over
// the particles, which are stored in cell order.  A thread's first particle
// is loaded before the grid-dependency wait: the particles were last written
// by the previous step's tracer, which belongs to an earlier graph launch
// (or an earlier, synchronised profiling step).
constexpr int TRACE_THREADS = 256;

__global__ void __launch_bounds__(TRACE_THREADS, 3) psf_trace(float4 *__restrict__ parts, long long P,
                                                 const int32_t *__restrict__ perm,
                                                 const float2 *__restrict__ pairs, GridDev g, TraceParams tp,
                                                 const unsigned long long *__restrict__ step_ctr)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float4 p = i < P ? parts[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    grid_dependency_wait();
    launch_dependents();
    const uint64_t step = *step_ctr - 1ull;
    for (bool first = true; i < P; i += stride, first = false) {
        if (!first) p = parts[i];
        parts[i] = advance_particle(p, g, pairs, tp, step, perm, (size_t)i);
    }
}

__global__ void psf_particle_keys(const float4 *__restrict__ in, long long P, GridDev g,
                                  uint32_t *__restrict__ keys, int32_t *__restrict__ idx)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const float4 p = in[i];
    const int x = clampi((int)floorf((p.x - g.mn[0]) * g.inv_h), 0, g.nx - 1);
    const int y = clampi((int)floorf((p.y - g.mn[1]) * g.inv_h), 0, g.ny - 1);
    const int z = clampi((int)floorf((p.z - g.mn[2]) * g.inv_h), 0, g.nz - 1);
    keys[i] = spread10((uint32_t)x) | (spread10((uint32_t)y) << 1) | (spread10((uint32_t)z) << 2);
    idx[i] = (int32_t)i;
}

__global__ void psf_gather_particles(const float4 *__restrict__ in, const int32_t *__restrict__ perm,
                                     float4 *__restrict__ out, long long P)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) out[i] = in[perm[i]];
}

__global__ void psf_scatter_particles(const float4 *__restrict__ in, const int32_t *__restrict__ perm,
                                      float4 *__restrict__ out, long long P)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) out[perm[i]] = in[i];
}

int sort_particles_temp_bytes(long long P, size_t *bytes)
{
    *bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, *bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                                    (const int32_t *)nullptr, (int32_t *)nullptr, (int)P);
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "cub sort sizing");
}

int launch_order_particles(const PlainDev &d, const OrderBufs &o, cudaStream_t st, bool resort)
{
    if (d.P == 0) return PSF_OK;
    const unsigned blocks = (unsigned)((d.P + 255) / 256);
    if (!resort) {  // keep the current order (perm) and only gather the new values into it
        psf_gather_particles<<<blocks, 256, 0, st>>>(o.staging, d.perm, d.parts, d.P);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? PSF_OK : cuda_fail(e, "particle gather launch");
    }
    psf_particle_keys<<<blocks, 256, 0, st>>>(o.staging, d.P, d.grid, o.keys_in, o.idx_in);
    size_t tmp = o.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(o.temp, tmp, o.keys_in, o.keys_out, o.idx_in,
                                                    const_cast<int32_t *>(d.perm),
                                                    (int)d.P, 0, 30, st);
    if (e != cudaSuccess) return cuda_fail(e, "cub sort");
    psf_gather_particles<<<blocks, 256, 0, st>>>(o.staging, d.perm, d.parts, d.P);
    e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "particle ordering launch");
}

int launch_unorder_particles(const PlainDev &d, const OrderBufs &o, cudaStream_t st)
{
    if (d.P == 0) return PSF_OK;
    const unsigned blocks = (unsigned)((d.P + 255) / 256);
    psf_scatter_particles<<<blocks, 256, 0, st>>>(d.parts, d.perm, o.staging, d.P);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "particle un-ordering launch");
}

// ------------------------------------------------------------- launchers
int launch_contract_state(const PlainDev &d, cudaStream_t st)
{
    const int CH = (d.Np + 127) / 128;
    const dim3 grid(d.N * d.S), block(256);
#define PSF_CASE(n)                                                                                   \
    case n:                                                                                           \
        psf_contract_state<n><<<grid, block, 0, st>>>(d.C, d.N, d.Np, d.S, d.w, d.w_next, d.dwpart,  \
                                                      d.lam, d.force, d.sp, d.ticket, d.step_ctr,    \
                                                      d.step_ctr_next);                              \
        break;
    switch (CH) {
        PSF_CASE(1)
        PSF_CASE(2)
        PSF_CASE(3)
        PSF_CASE(4)
        PSF_CASE(5)
        PSF_CASE(6)
        PSF_CASE(7)
        PSF_CASE(8)
    default:
        return fail(PSF_ERR_UNSUPPORTED, "mode count above the supported maximum");
    }
#undef PSF_CASE
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_contract_state launch");
}


// Launch configuration of a step kernel that may start while the previous
// kernel in the stream finishes (programmatic stream serialisation).
struct PdlLaunch {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    PdlLaunch(unsigned grid, unsigned block, cudaStream_t st)
    {
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(block);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
};

int launch_reconstruct(const PlainDev &d, cudaStream_t st, bool after_kernel)
{
    const long long blocks = (d.n_active + 127) / 128;
    PdlLaunch L((unsigned)blocks, 256, st);
    if (!after_kernel) L.cfg.numAttrs = 0;
    cudaError_t e = cudaLaunchKernelEx(&L.cfg, psf_reconstruct, (const float *)d.phiT, (long long)d.ldp,
                                       (const int32_t *)d.faces, (long long)d.n_active, (int)d.N, (const double *)d.w,
                                       d.u, reinterpret_cast<float *>(d.pairs), (const int32_t *)d.pair_dst);
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_reconstruct launch");
}

int trace_blocks_per_sm()
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psf_trace, TRACE_THREADS, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 4;
    return per_sm;
}

int launch_trace(const PlainDev &d, cudaStream_t st, bool after_kernel)
{
    if (d.P == 0) return PSF_OK;
    const long long blocks =
        std::min<long long>((d.P + TRACE_THREADS - 1) / TRACE_THREADS, std::max(1, d.trace_blocks));
    PdlLaunch L((unsigned)blocks, TRACE_THREADS, st);
    if (!after_kernel) L.cfg.numAttrs = 0;
    cudaError_t e = cudaLaunchKernelEx(&L.cfg, psf_trace, d.parts, (long long)d.P, (const int32_t *)d.perm,
                                       d.trace_pairs, d.grid, d.tp, d.trace_ctr);
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_trace launch");
}

}  // namespace psf
