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
//   2. psf_reconstruct     u = Phi w with Phi stored mode-major (faces
//      contiguous, the tracer's face signs folded in), so every warp streams
//      512 contiguous bytes per mode; scatter to the reference face numbering.
//      (replaces simulation.cl:313-354)
//   3. psf_trace           one thread per particle, trilinear staggered
//      interpolation from the signed face field, RK1 or RK4, box clamp,
//      lifetime and respawn.  (replaces simulation.cl:33-205)

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

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }
__device__ __forceinline__ float mixf(float x, float y, float a) { return x * (1.f - a) + y * a; }

__device__ __forceinline__ uint32_t zface(const GridDev &g, int x, int y, int z)
{
    return (uint32_t)z * (uint32_t)(g.nx * g.ny) + (uint32_t)(y * g.nx + x);
}
__device__ __forceinline__ uint32_t yface(const GridDev &g, int x, int y, int z)
{
    return (uint32_t)z * (uint32_t)((g.ny + 1) * g.nx) + (uint32_t)(y * g.nx + x) + g.yoff;
}
__device__ __forceinline__ uint32_t xface(const GridDev &g, int x, int y, int z)
{
    return (uint32_t)z * (uint32_t)(g.ny * (g.nx + 1)) + (uint32_t)(y * (g.nx + 1) + x) + g.xoff;
}

// Counter-based generator for respawns (SplitMix64 output function); the
// oracle uses the same function so respawns are reproducible.
__host__ __device__ __forceinline__ uint32_t respawn_hash(uint64_t seed, uint64_t step, uint32_t idx,
                                                          uint32_t k)
{
    uint64_t x = seed ^ (step * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)idx << 32) ^
                 ((uint64_t)k * 0xD1B54A32D192ED03ull);
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (uint32_t)(x >> 32);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum over 256 threads; result valid in every thread.
__device__ double block_sum_256(double v, double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) t += red[i];
    return t;
}

// ------------------------------------------------------- 1. contraction
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

// ---------------------------------------------------- 2. reconstruction
// 256 threads = 8 warps x 32 lanes; a block covers 128 consecutive active
// faces (4 per lane, one float4 per mode); warp g sums modes i = g (mod 8).
__global__ void __launch_bounds__(256) psf_reconstruct(const float *__restrict__ phiT, long long ldp,
                                                       const int32_t *__restrict__ faces, long long n_active,
                                                       int N, const double *__restrict__ w, float *__restrict__ u)
{
    __shared__ float wsm[PSF_MAX_MODES];
    __shared__ float4 red[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < N; i += 256) wsm[i] = (float)w[i];
    __syncthreads();
    const long long f0 = (long long)blockIdx.x * 128 + lane * 4;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (f0 < ldp) {
        const float *base = phiT + f0;
#pragma unroll 4
        for (int i = warp; i < N; i += 8) {
            const float4 v = __ldg(reinterpret_cast<const float4 *>(base + (size_t)i * ldp));
            const float wi = wsm[i];
            acc.x = fmaf(v.x, wi, acc.x);
            acc.y = fmaf(v.y, wi, acc.y);
            acc.z = fmaf(v.z, wi, acc.z);
            acc.w = fmaf(v.w, wi, acc.w);
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
        for (int q = 0; q < 4; ++q)
            if (f0 + q < n_active) u[faces[f0 + q]] = vals[q];
    }
}

// --------------------------------------------------------- 3. tracing
// Staggered trilinear interpolation (psfsolver.cpp:80-212): for each
// component, eight face samples mixed along y, then x, then z.  The face
// field is already signed, so no sign-string lookups are needed.
__device__ __forceinline__ float3 velocity_at(const GridDev &g, const float *__restrict__ u, float px, float py,
                                              float pz)
{
    const float gix = (g.shift[0] + px) * g.inv_h;
    const float giy = (g.shift[1] + py) * g.inv_h;
    const float giz = (g.shift[2] + pz) * g.inv_h;
    const float gwx = (px - g.mn[0]) * g.inv_h;
    const float gwy = (py - g.mn[1]) * g.inv_h;
    const float gwz = (pz - g.mn[2]) * g.inv_h;
    const int xO = clampi((int)floorf(gix), 0, g.nx - 1);
    const int yO = clampi((int)floorf(giy), 0, g.ny - 1);
    const int zO = clampi((int)floorf(giz), 0, g.nz - 1);
    const int xr = (int)floorf(gix - 0.5f), yr = (int)floorf(giy - 0.5f), zr = (int)floorf(giz - 0.5f);
    const int xM = clampi(xr, 0, g.nx - 1), xP = clampi(xr + 1, 0, g.nx - 1);
    const int yM = clampi(yr, 0, g.ny - 1), yP = clampi(yr + 1, 0, g.ny - 1);
    const int zM = clampi(zr, 0, g.nz - 1), zP = clampi(zr + 1, 0, g.nz - 1);
    float3 v;
    {  // x: faces (xO | xO+1, yM | yP, zM | zP)
        const float tx = gwx - (float)xO, ty = gwy - ((float)yM + 0.5f), tz = gwz - ((float)zM + 0.5f);
        const uint32_t i00 = xface(g, xO, yM, zM), i10 = xface(g, xO, yP, zM);
        const uint32_t i01 = xface(g, xO, yM, zP), i11 = xface(g, xO, yP, zP);
        const float a = mixf(__ldg(u + i00), __ldg(u + i10), ty);
        const float b = mixf(__ldg(u + i00 + 1), __ldg(u + i10 + 1), ty);
        const float c = mixf(__ldg(u + i01), __ldg(u + i11), ty);
        const float d = mixf(__ldg(u + i01 + 1), __ldg(u + i11 + 1), ty);
        v.x = mixf(mixf(a, b, tx), mixf(c, d, tx), tz);
    }
    {  // y: faces (xM | xP, yO | yO+1, zM | zP)
        const float tx = gwx - ((float)xM + 0.5f), ty = gwy - (float)yO, tz = gwz - ((float)zM + 0.5f);
        const uint32_t iM0 = yface(g, xM, yO, zM), iP0 = yface(g, xP, yO, zM);
        const uint32_t iM1 = yface(g, xM, yO, zP), iP1 = yface(g, xP, yO, zP);
        const uint32_t up = (uint32_t)g.nx;  // yO + 1
        const float a = mixf(__ldg(u + iM0), __ldg(u + iM0 + up), ty);
        const float b = mixf(__ldg(u + iP0), __ldg(u + iP0 + up), ty);
        const float c = mixf(__ldg(u + iM1), __ldg(u + iM1 + up), ty);
        const float d = mixf(__ldg(u + iP1), __ldg(u + iP1 + up), ty);
        v.y = mixf(mixf(a, b, tx), mixf(c, d, tx), tz);
    }
    {  // z: faces (xM | xP, yM | yP, zO | zO+1)
        const float tx = gwx - ((float)xM + 0.5f), ty = gwy - ((float)yM + 0.5f), tz = gwz - (float)zO;
        const uint32_t iMM = zface(g, xM, yM, zO), iMP = zface(g, xM, yP, zO);
        const uint32_t iPM = zface(g, xP, yM, zO), iPP = zface(g, xP, yP, zO);
        const uint32_t up = (uint32_t)(g.nx * g.ny);  // zO + 1
        const float a = mixf(__ldg(u + iMM), __ldg(u + iMP), ty);
        const float b = mixf(__ldg(u + iPM), __ldg(u + iPP), ty);
        const float c = mixf(__ldg(u + iMM + up), __ldg(u + iMP + up), ty);
        const float d = mixf(__ldg(u + iPM + up), __ldg(u + iPP + up), ty);
        v.z = mixf(mixf(a, b, tx), mixf(c, d, tx), tz);
    }
    return v;
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

__global__ void __launch_bounds__(256) psf_trace(float4 *__restrict__ parts, long long P,
                                                 const int32_t *__restrict__ perm,
                                                 const float *__restrict__ u, GridDev g, TraceParams tp,
                                                 const unsigned long long *__restrict__ step_ctr)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    float4 p = parts[i];
    if (p.w > 0.f) {
        const float dt = tp.dt;
        float3 v;
        if (tp.rk4) {
            const float3 k1 = velocity_at(g, u, p.x, p.y, p.z);
            float qx = clampf(p.x + 0.5f * dt * k1.x, g.mn[0], g.mx[0]);
            float qy = clampf(p.y + 0.5f * dt * k1.y, g.mn[1], g.mx[1]);
            float qz = clampf(p.z + 0.5f * dt * k1.z, g.mn[2], g.mx[2]);
            const float3 k2 = velocity_at(g, u, qx, qy, qz);
            qx = clampf(p.x + 0.5f * dt * k2.x, g.mn[0], g.mx[0]);
            qy = clampf(p.y + 0.5f * dt * k2.y, g.mn[1], g.mx[1]);
            qz = clampf(p.z + 0.5f * dt * k2.z, g.mn[2], g.mx[2]);
            const float3 k3 = velocity_at(g, u, qx, qy, qz);
            qx = clampf(p.x + dt * k3.x, g.mn[0], g.mx[0]);
            qy = clampf(p.y + dt * k3.y, g.mn[1], g.mx[1]);
            qz = clampf(p.z + dt * k3.z, g.mn[2], g.mx[2]);
            const float3 k4 = velocity_at(g, u, qx, qy, qz);
            v.x = (k1.x + 2.f * k2.x + 2.f * k3.x + k4.x) / 6.f;
            v.y = (k1.y + 2.f * k2.y + 2.f * k3.y + k4.y) / 6.f;
            v.z = (k1.z + 2.f * k2.z + 2.f * k3.z + k4.z) / 6.f;
        } else {
            v = velocity_at(g, u, p.x, p.y, p.z);
        }
        p.x = clampf(p.x + dt * v.x, g.mn[0], g.mx[0]);
        p.y = clampf(p.y + dt * v.y, g.mn[1], g.mx[1]);
        p.z = clampf(p.z + dt * v.z, g.mn[2], g.mx[2]);
        p.w = p.w - 1.f;
    } else {
        // psfsolver.cpp:217-222 with the counter-based generator.
        // Particles are stored in cell order; the generator is keyed by the
        // caller's particle index so respawns do not depend on that order.
        const uint64_t step = *step_ctr - 1ull;
        const uint32_t id = (uint32_t)perm[i];
        const uint32_t r1 = respawn_hash(tp.seed, step, id, 1) % 1024u;
        const uint32_t r2 = respawn_hash(tp.seed, step, id, 2) % 1024u;
        const uint32_t r3 = respawn_hash(tp.seed, step, id, 3) % 1024u;
        const float cz = g.mn[2] + 0.5f * (g.mx[2] - g.mn[2]);
        p.x = (float)(((double)r1 / 1024.0 - 0.5) * 0.25);
        p.y = g.mn[1] + 0.2f;
        p.z = (float)(-(double)cz + ((double)r3 / 1024.0 - 0.5) * 0.25);
        p.w = (float)((double)tp.lifetime * ((double)r2 / 1024.0));
    }
    parts[i] = p;
}

// ------------------------------------------------------- particle order
// Particles are kept sorted by the Morton code of their voxel so that the
// threads of a warp gather from a few neighbouring cells of the face field.
__device__ __forceinline__ uint32_t spread10(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
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

int launch_reconstruct(const PlainDev &d, cudaStream_t st)
{
    const long long blocks = (d.n_active + 127) / 128;
    psf_reconstruct<<<(unsigned)blocks, 256, 0, st>>>(d.phiT, d.ldp, d.faces, d.n_active, d.N, d.w, d.u);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_reconstruct launch");
}

int launch_trace(const PlainDev &d, cudaStream_t st)
{
    if (d.P == 0) return PSF_OK;
    const long long blocks = (d.P + 255) / 256;
    psf_trace<<<(unsigned)blocks, 256, 0, st>>>(d.parts, d.P, d.perm, d.u, d.grid, d.tp, d.step_ctr);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSF_OK : cuda_fail(e, "psf_trace launch");
}

}  // namespace psf
