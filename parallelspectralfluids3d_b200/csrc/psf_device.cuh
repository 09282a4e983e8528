// Device helpers shared by the single-instance and the batched kernels:
// reference face numbering, the staggered trilinear interpolant, one
// particle step, the respawn generator, Morton keys and FP64 reductions.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "psf_b200.h"
#include "psf_internal.h"

namespace psf {

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
__device__ inline double block_sum_256(double v, double *red)
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

// One particle step (psfsolver.cpp:75-224): RK1 or RK4 with the box clamp
// on every stage, lifetime decrement, and respawn from the counter-based
// generator keyed by the caller-order index `id` when the lifetime ran out.
// `step` is the index of the step being taken (0 for the first).
__device__ __forceinline__ float4 advance_particle(float4 p, const GridDev &g, const float *__restrict__ u,
                                                   const TraceParams &tp, uint64_t step, uint32_t id)
{
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
        const uint32_t r1 = respawn_hash(tp.seed, step, id, 1) % 1024u;
        const uint32_t r2 = respawn_hash(tp.seed, step, id, 2) % 1024u;
        const uint32_t r3 = respawn_hash(tp.seed, step, id, 3) % 1024u;
        const float cz = g.mn[2] + 0.5f * (g.mx[2] - g.mn[2]);
        p.x = (float)(((double)r1 / 1024.0 - 0.5) * 0.25);
        p.y = g.mn[1] + 0.2f;
        p.z = (float)(-(double)cz + ((double)r3 / 1024.0 - 0.5) * 0.25);
        p.w = (float)((double)tp.lifetime * ((double)r2 / 1024.0));
    }
    return p;
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

}  // namespace psf
