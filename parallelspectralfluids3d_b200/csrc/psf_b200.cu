// B200 (sm_100a) spectral-fluid step engine: kernels and the C ABI of
// include/psf_b200.h for single-instance contexts.
//
// One step (the reference's PSFSolver::integrate, Solver/SolverImpl/
// psfsolver.cpp:21-234) is two kernels, captured once into a CUDA graph: the
// coefficient half (contraction, FP64 state update, reconstruction) in
// psf_plain_tma.cu, then
//
//   psf_trace   one thread per particle, trilinear staggered interpolation
//               from the signed face field, RK1 or RK4, box clamp, lifetime
//               and respawn.  (replaces simulation.cl:33-205)
//
// This file also holds the particle ordering kernels, the error helpers and
// psf_contract_state, the staging-free contraction + state update that the
// allocation-free entry point runs.

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

// ------------------------------------------- contraction without staging
// Contraction + FP64 state update with plain 128-bit loads and no tensor
// maps; psf_coeff_step_static (psf_noalloc.cu) runs it on caller buffers.
// Block b handles mode k = b / S and row slice s = b % S of C_k.  Lane l of a
// warp owns columns [4l + 128c, 4l + 128c + 4) for c < CH, with w_j in
// registers; warps walk rows a.  Each lane accumulates
// sum_a w_a * (C[k][a][j..j+3] . w[j..j+3]) in FP64, so no per-row reduction
// is needed; one block reduction at the end.
template <int CH>
__global__ void __launch_bounds__(256) psf_contract_state(const float *__restrict__ C, int N, int Np, int S,
                                                          double *__restrict__ w, double *__restrict__ dwpart,
                                                          const double *__restrict__ lam,
                                                          const double *__restrict__ force, StateParams sp,
                                                          unsigned int *__restrict__ ticket,
                                                          unsigned long long *__restrict__ step_ctr)
{
    __shared__ double red[8];
    __shared__ int is_last;
    __shared__ double wnew[PSF_MAX_MODES];

    const int k = blockIdx.x / S;
    const int s = blockIdx.x - k * S;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    float wj[CH][4];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int col = c * 128 + lane * 4 + q;
            wj[c][q] = col < N ? (float)w[col] : 0.f;
        }
    }
    const int rows = (N + S - 1) / S;
    const int a0 = s * rows;
    const int a1 = min(N, a0 + rows);
    const float *Ck = C + (size_t)k * N * Np;
    double acc = 0.0;
#pragma unroll 4
    for (int a = a0 + warp; a < a1; a += 8) {
        const float4 *row = reinterpret_cast<const float4 *>(Ck + (size_t)a * Np);
        float part = 0.f;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            if (c * 128 + lane * 4 < Np) {
                const float4 v = __ldg(row + c * 32 + lane);
                part = fmaf(v.x, wj[c][0], part);
                part = fmaf(v.y, wj[c][1], part);
                part = fmaf(v.z, wj[c][2], part);
                part = fmaf(v.w, wj[c][3], part);
            }
        }
        acc = fma(w[a], (double)part, acc);
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
        const double wi = w[i];
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
        w[i] = v;
    }
    if (threadIdx.x == 0) {
        *ticket = 0u;
        *step_ctr += 1ull;
    }
}


// Persistent grid (a whole number of resident blocks per SM) striding over
// the particles, which are stored in cell order.
__global__ void __launch_bounds__(256, 3) psf_trace(float4 *__restrict__ parts, long long P,
                                                 const int32_t *__restrict__ perm,
                                                 const float2 *__restrict__ pairs, GridDev g, TraceParams tp,
                                                 const unsigned long long *__restrict__ step_ctr)
{
    const uint64_t step = *step_ctr - 1ull;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += stride) {
        float4 p = parts[i];
        p = advance_particle(p, g, pairs, tp, step, perm, (size_t)i);
        parts[i] = p;
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

int launch_order_particles(const PlainDev &d, const OrderBufs &o, cudaStream_t st)
{
    if (d.P == 0) return PSF_OK;
    const unsigned blocks = (unsigned)((d.P + 255) / 256);
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
// ------------------------------------------------------------- launchers
int launch_contract_state(const PlainDev &d, cudaStream_t st)
{
    const int CH = (d.Np + 127) / 128;
    const dim3 grid(d.N * d.S), block(256);
#define PSF_CASE(n)                                                                                   \
    case n:                                                                                           \
        psf_contract_state<n><<<grid, block, 0, st>>>(d.C, d.N, d.Np, d.S, d.w, d.dwpart, d.lam,     \
                                                      d.force, d.sp, d.ticket, d.step_ctr);          \
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


int trace_blocks_per_sm()
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psf_trace, 256, 0) != cudaSuccess || per_sm < 1)
        per_sm = 4;
    return per_sm;
}

int launch_trace(const PlainDev &d, cudaStream_t st)
{
    if (d.P == 0) return PSF_OK;
    const long long blocks = std::min<long long>((d.P + 255) / 256, std::max(1, d.trace_blocks));
    psf_trace<<<(unsigned)blocks, 256, 0, st>>>(d.parts, d.P, d.perm, d.pairs, d.grid, d.tp, d.step_ctr);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_trace launch");
}

}  // namespace psf
