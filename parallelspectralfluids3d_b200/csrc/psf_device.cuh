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
// glm::mix(x, y, a) = x (1 - a) + y a, evaluated as x + a (y - x) (one FMA).
__device__ __forceinline__ float mixf(float x, float y, float a) { return fmaf(a, y - x, x); }

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

// ------------------------------------------------------------------ tracing
// The tracer reads the face field through a per-voxel copy ("face pairs"):
// for voxel v, pairs[v] = (u of its x-face at x, at x+1), pairs[V + v] the
// same for y, pairs[2V + v] for z, already carrying the tracer's face signs.
// One trilinear component then needs four aligned float2 loads instead of
// eight scalar gathers.  The interpolant is the reference's
// (psfsolver.cpp:80-212): clamped staggered cell indices, eight face samples
// per component mixed along y, then x, then z, weights not clamped.
__device__ __forceinline__ uint32_t voxel(const GridDev &g, int x, int y, int z)
{
    return (uint32_t)z * (uint32_t)(g.nx * g.ny) + (uint32_t)(y * g.nx + x);
}

// Staggered cell of a position: the clamped voxel indices of the three
// component stencils, and the position in voxel units from the box corner.
// `key` packs the unclamped floor indices they all derive from, so two
// positions share a cell exactly when their keys are equal.
struct Cell {
    int xO, yO, zO, xM, xP, yM, yP, zM, zP;
    uint32_t keyO, keyR;
};

__device__ __forceinline__ Cell cell_of(const GridDev &g, float px, float py, float pz, float3 &gw)
{
    const float gix = (g.shift[0] + px) * g.inv_h;
    const float giy = (g.shift[1] + py) * g.inv_h;
    const float giz = (g.shift[2] + pz) * g.inv_h;
    gw.x = (px - g.mn[0]) * g.inv_h;
    gw.y = (py - g.mn[1]) * g.inv_h;
    gw.z = (pz - g.mn[2]) * g.inv_h;
    Cell c;
    c.xO = clampi(__float2int_rd(gix), 0, g.nx - 1);
    c.yO = clampi(__float2int_rd(giy), 0, g.ny - 1);
    c.zO = clampi(__float2int_rd(giz), 0, g.nz - 1);
    const int xr = __float2int_rd(gix - 0.5f), yr = __float2int_rd(giy - 0.5f), zr = __float2int_rd(giz - 0.5f);
    c.xM = clampi(xr, 0, g.nx - 1);
    c.xP = clampi(xr + 1, 0, g.nx - 1);
    c.yM = clampi(yr, 0, g.ny - 1);
    c.yP = clampi(yr + 1, 0, g.ny - 1);
    c.zM = clampi(zr, 0, g.nz - 1);
    c.zP = clampi(zr + 1, 0, g.nz - 1);
    // Clamped indices are in [0, 1023] and xr + 1 in [0, 1024): 10 bits each.
    c.keyO = (uint32_t)c.xO | ((uint32_t)c.yO << 10) | ((uint32_t)c.zO << 20);
    c.keyR = (uint32_t)clampi(xr + 1, 0, 1023) | ((uint32_t)clampi(yr + 1, 0, 1023) << 10) |
             ((uint32_t)clampi(zr + 1, 0, 1023) << 20);
    return c;
}

__device__ __forceinline__ bool same_cell(const Cell &a, const Cell &b)
{
    return a.keyO == b.keyO && a.keyR == b.keyR;
}

// The 24 face samples of a cell as 12 face pairs.
struct CellSamples {
    float2 x00, x10, x01, x11;  // x-face pairs at (xO, yM|yP, zM|zP)
    float2 yM0, yP0, yM1, yP1;  // y-face pairs at (xM|xP, yO, zM|zP)
    float2 zMM, zMP, zPM, zPP;  // z-face pairs at (xM|xP, yM|yP, zO)
};

__device__ __forceinline__ void gather_cell(const GridDev &g, const float2 *__restrict__ pairs, const Cell &c,
                                            CellSamples &s)
{
    const uint32_t V = (uint32_t)g.nx * (uint32_t)g.ny * (uint32_t)g.nz;
    const float2 *__restrict__ pxp = pairs;
    const float2 *__restrict__ pyp = pairs + V;
    const float2 *__restrict__ pzp = pairs + 2 * (size_t)V;
    s.x00 = __ldg(pxp + voxel(g, c.xO, c.yM, c.zM));
    s.x10 = __ldg(pxp + voxel(g, c.xO, c.yP, c.zM));
    s.x01 = __ldg(pxp + voxel(g, c.xO, c.yM, c.zP));
    s.x11 = __ldg(pxp + voxel(g, c.xO, c.yP, c.zP));
    s.yM0 = __ldg(pyp + voxel(g, c.xM, c.yO, c.zM));
    s.yP0 = __ldg(pyp + voxel(g, c.xP, c.yO, c.zM));
    s.yM1 = __ldg(pyp + voxel(g, c.xM, c.yO, c.zP));
    s.yP1 = __ldg(pyp + voxel(g, c.xP, c.yO, c.zP));
    s.zMM = __ldg(pzp + voxel(g, c.xM, c.yM, c.zO));
    s.zMP = __ldg(pzp + voxel(g, c.xM, c.yP, c.zO));
    s.zPM = __ldg(pzp + voxel(g, c.xP, c.yM, c.zO));
    s.zPP = __ldg(pzp + voxel(g, c.xP, c.yP, c.zO));
}

__device__ __forceinline__ float3 interpolate(const Cell &c, const CellSamples &s, const float3 &gw)
{
    float3 v;
    {  // x: faces (xO | xO+1, yM | yP, zM | zP)
        const float tx = gw.x - (float)c.xO, ty = gw.y - ((float)c.yM + 0.5f), tz = gw.z - ((float)c.zM + 0.5f);
        const float a = mixf(s.x00.x, s.x10.x, ty);
        const float b = mixf(s.x00.y, s.x10.y, ty);
        const float cc = mixf(s.x01.x, s.x11.x, ty);
        const float d = mixf(s.x01.y, s.x11.y, ty);
        v.x = mixf(mixf(a, b, tx), mixf(cc, d, tx), tz);
    }
    {  // y: faces (xM | xP, yO | yO+1, zM | zP)
        const float tx = gw.x - ((float)c.xM + 0.5f), ty = gw.y - (float)c.yO, tz = gw.z - ((float)c.zM + 0.5f);
        const float a = mixf(s.yM0.x, s.yM0.y, ty);
        const float b = mixf(s.yP0.x, s.yP0.y, ty);
        const float cc = mixf(s.yM1.x, s.yM1.y, ty);
        const float d = mixf(s.yP1.x, s.yP1.y, ty);
        v.y = mixf(mixf(a, b, tx), mixf(cc, d, tx), tz);
    }
    {  // z: faces (xM | xP, yM | yP, zO | zO+1)
        const float tx = gw.x - ((float)c.xM + 0.5f), ty = gw.y - ((float)c.yM + 0.5f), tz = gw.z - (float)c.zO;
        const float a = mixf(s.zMM.x, s.zMP.x, ty);
        const float b = mixf(s.zPM.x, s.zPP.x, ty);
        const float cc = mixf(s.zMM.y, s.zMP.y, ty);
        const float d = mixf(s.zPM.y, s.zPP.y, ty);
        v.z = mixf(mixf(a, b, tx), mixf(cc, d, tx), tz);
    }
    return v;
}

// Velocity at a position; `c`/`s` carry the last gathered cell, and the
// samples are loaded again only when the position lies in another cell.
__device__ __forceinline__ float3 velocity_cached(const GridDev &g, const float2 *__restrict__ pairs, float px,
                                                  float py, float pz, Cell &c, CellSamples &s, bool &have)
{
    float3 gw;
    const Cell n = cell_of(g, px, py, pz, gw);
    if (!have || !same_cell(n, c)) {
        c = n;
        gather_cell(g, pairs, c, s);
        have = true;
    }
    return interpolate(c, s, gw);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// One particle step (psfsolver.cpp:75-224): RK1 or RK4 with the box clamp
// on every stage, lifetime decrement, and respawn from the counter-based
// generator keyed by the caller-order index `id` when the lifetime ran out.
// `step` is the index of the step being taken (0 for the first).
__device__ __forceinline__ float4 advance_particle(float4 p, const GridDev &g, const float2 *__restrict__ u,
                                                   const TraceParams &tp, uint64_t step, uint32_t id)
{
    if (p.w > 0.f) {
        const float dt = tp.dt;
        Cell c;
        CellSamples cs;
        bool have = false;
        float3 v;
        if (tp.rk4) {
            const float3 k1 = velocity_cached(g, u, p.x, p.y, p.z, c, cs, have);
            float qx = clampf(p.x + 0.5f * dt * k1.x, g.mn[0], g.mx[0]);
            float qy = clampf(p.y + 0.5f * dt * k1.y, g.mn[1], g.mx[1]);
            float qz = clampf(p.z + 0.5f * dt * k1.z, g.mn[2], g.mx[2]);
            const float3 k2 = velocity_cached(g, u, qx, qy, qz, c, cs, have);
            qx = clampf(p.x + 0.5f * dt * k2.x, g.mn[0], g.mx[0]);
            qy = clampf(p.y + 0.5f * dt * k2.y, g.mn[1], g.mx[1]);
            qz = clampf(p.z + 0.5f * dt * k2.z, g.mn[2], g.mx[2]);
            const float3 k3 = velocity_cached(g, u, qx, qy, qz, c, cs, have);
            qx = clampf(p.x + dt * k3.x, g.mn[0], g.mx[0]);
            qy = clampf(p.y + dt * k3.y, g.mn[1], g.mx[1]);
            qz = clampf(p.z + dt * k3.z, g.mn[2], g.mx[2]);
            const float3 k4 = velocity_cached(g, u, qx, qy, qz, c, cs, have);
            v.x = (k1.x + 2.f * k2.x + 2.f * k3.x + k4.x) / 6.f;
            v.y = (k1.y + 2.f * k2.y + 2.f * k3.y + k4.y) / 6.f;
            v.z = (k1.z + 2.f * k2.z + 2.f * k3.z + k4.z) / 6.f;
        } else {
            v = velocity_cached(g, u, p.x, p.y, p.z, c, cs, have);
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
