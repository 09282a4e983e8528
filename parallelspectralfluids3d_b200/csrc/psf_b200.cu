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
