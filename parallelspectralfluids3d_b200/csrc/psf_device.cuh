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

// Staggered cell of a position.  Every index the three component stencils
// use derives from k = floor(2 * gi) per axis (gi = the reference's index
// coordinate): floor(gi) = k >> 1 and floor(gi - 1/2) = (k - 1) >> 1, the
// latter exact because gi - 1/2 is exact in FP32 wherever the clamp to the
// grid does not decide the index anyway.  Two positions share a cell when
// their k, clamped to [-1, 2n], agree: the key packs those.
__device__ __forceinline__ unsigned long long cell_key(const GridDev &g, float px, float py, float pz, int &kx,
                                                       int &ky, int &kz)
{
    const float gix = (g.shift[0] + px) * g.inv_h;
    const float giy = (g.shift[1] + py) * g.inv_h;
    const float giz = (g.shift[2] + pz) * g.inv_h;
    kx = clampi(__float2int_rd(2.0f * gix), -1, 2 * g.nx);
    ky = clampi(__float2int_rd(2.0f * giy), -1, 2 * g.ny);
    kz = clampi(__float2int_rd(2.0f * giz), -1, 2 * g.nz);
    return (unsigned long long)(uint32_t)(kx + 1) | ((unsigned long long)(uint32_t)(ky + 1) << 21) |
           ((unsigned long long)(uint32_t)(kz + 1) << 42);
}

// The gathered cell: stencil origins as floats and the 24 face samples as 12
// face pairs, each second sample of a lerp stored as its difference to the
// first (mixf(x, y, t) = fma(t, y - x, x) then costs one FMA).
struct CellCache {
    int kx, ky, kz;        // the cell: floor(2 gi) per axis, clamped to [-1, 2n]
    float oxO, oyO, ozO;   // xO, yO, zO
    float oxM, oyM, ozM;   // xM + 1/2, yM + 1/2, zM + 1/2
    float2 x00, dx10, x01, dx11;  // x faces at (xO, yM|yP, zM|zP), differences along y
    float2 yM0, yP0, yM1, yP1;    // y face pairs at (xM|xP, yO, zM|zP), .y = difference along y
    float2 zMM, dzMP, zPM, dzPP;  // z faces at (xM|xP, yM|yP, zO), differences along y
};

__device__ __forceinline__ void gather_cell(const GridDev &g, const float2 *__restrict__ pairs, int kx, int ky,
                                            int kz, CellCache &c)
{
    const int xO = clampi(kx >> 1, 0, g.nx - 1), yO = clampi(ky >> 1, 0, g.ny - 1), zO = clampi(kz >> 1, 0, g.nz - 1);
    const int xr = (kx - 1) >> 1, yr = (ky - 1) >> 1, zr = (kz - 1) >> 1;
    const int xM = clampi(xr, 0, g.nx - 1), xP = clampi(xr + 1, 0, g.nx - 1);
    const int yM = clampi(yr, 0, g.ny - 1), yP = clampi(yr + 1, 0, g.ny - 1);
    const int zM = clampi(zr, 0, g.nz - 1), zP = clampi(zr + 1, 0, g.nz - 1);
    c.oxO = (float)xO;
    c.oyO = (float)yO;
    c.ozO = (float)zO;
    c.oxM = (float)xM + 0.5f;
    c.oyM = (float)yM + 0.5f;
    c.ozM = (float)zM + 0.5f;
    const uint32_t V = (uint32_t)g.nx * (uint32_t)g.ny * (uint32_t)g.nz;
    const float2 *__restrict__ pxp = pairs;
    const float2 *__restrict__ pyp = pairs + V;
    const float2 *__restrict__ pzp = pairs + 2 * (size_t)V;
    const float2 x00 = __ldg(pxp + voxel(g, xO, yM, zM));
    const float2 x10 = __ldg(pxp + voxel(g, xO, yP, zM));
    const float2 x01 = __ldg(pxp + voxel(g, xO, yM, zP));
    const float2 x11 = __ldg(pxp + voxel(g, xO, yP, zP));
    const float2 yM0 = __ldg(pyp + voxel(g, xM, yO, zM));
    const float2 yP0 = __ldg(pyp + voxel(g, xP, yO, zM));
    const float2 yM1 = __ldg(pyp + voxel(g, xM, yO, zP));
    const float2 yP1 = __ldg(pyp + voxel(g, xP, yO, zP));
    const float2 zMM = __ldg(pzp + voxel(g, xM, yM, zO));
    const float2 zMP = __ldg(pzp + voxel(g, xM, yP, zO));
    const float2 zPM = __ldg(pzp + voxel(g, xP, yM, zO));
    const float2 zPP = __ldg(pzp + voxel(g, xP, yP, zO));
    c.x00 = x00;
    c.dx10 = make_float2(x10.x - x00.x, x10.y - x00.y);
    c.x01 = x01;
    c.dx11 = make_float2(x11.x - x01.x, x11.y - x01.y);
    c.yM0 = make_float2(yM0.x, yM0.y - yM0.x);
    c.yP0 = make_float2(yP0.x, yP0.y - yP0.x);
    c.yM1 = make_float2(yM1.x, yM1.y - yM1.x);
    c.yP1 = make_float2(yP1.x, yP1.y - yP1.x);
    c.zMM = zMM;
    c.dzMP = make_float2(zMP.x - zMM.x, zMP.y - zMM.y);
    c.zPM = zPM;
    c.dzPP = make_float2(zPP.x - zPM.x, zPP.y - zPM.y);
}

__device__ __forceinline__ float3 interpolate(const CellCache &c, const float3 &gw)
{
    float3 v;
    {  // x: faces (xO | xO+1, yM | yP, zM | zP)
        const float tx = gw.x - c.oxO, ty = gw.y - c.oyM, tz = gw.z - c.ozM;
        const float a = fmaf(ty, c.dx10.x, c.x00.x);
        const float b = fmaf(ty, c.dx10.y, c.x00.y);
        const float cc = fmaf(ty, c.dx11.x, c.x01.x);
        const float d = fmaf(ty, c.dx11.y, c.x01.y);
        v.x = mixf(mixf(a, b, tx), mixf(cc, d, tx), tz);
    }
    {  // y: faces (xM | xP, yO | yO+1, zM | zP)
        const float tx = gw.x - c.oxM, ty = gw.y - c.oyO, tz = gw.z - c.ozM;
        const float a = fmaf(ty, c.yM0.y, c.yM0.x);
        const float b = fmaf(ty, c.yP0.y, c.yP0.x);
        const float cc = fmaf(ty, c.yM1.y, c.yM1.x);
        const float d = fmaf(ty, c.yP1.y, c.yP1.x);
        v.y = mixf(mixf(a, b, tx), mixf(cc, d, tx), tz);
    }
    {  // z: faces (xM | xP, yM | yP, zO | zO+1)
        const float tx = gw.x - c.oxM, ty = gw.y - c.oyM, tz = gw.z - c.ozO;
        const float a = fmaf(ty, c.dzMP.x, c.zMM.x);
        const float b = fmaf(ty, c.dzPP.x, c.zPM.x);
        const float cc = fmaf(ty, c.dzMP.y, c.zMM.y);
        const float d = fmaf(ty, c.dzPP.y, c.zPM.y);
        v.z = mixf(mixf(a, b, tx), mixf(cc, d, tx), tz);
    }
    return v;
}

// Velocity at a position; `c` carries the last gathered cell, and the
// samples are loaded again only when the position lies in another cell.
// When the box is centred (shift == -mn exactly, as for every domain built
// here) the reference's index coordinate (shift + p) / h and the weight
// coordinate (p - mn) / h are the same float, so it is computed once.
__device__ __forceinline__ float3 velocity_cached(const GridDev &g, const float2 *__restrict__ pairs, float px,
                                                  float py, float pz, CellCache &c, bool &have)
{
    float3 gw;
    gw.x = (px - g.mn[0]) * g.inv_h;
    gw.y = (py - g.mn[1]) * g.inv_h;
    gw.z = (pz - g.mn[2]) * g.inv_h;
    int kx, ky, kz;
    if (g.centered) {
        kx = clampi(__float2int_rd(2.0f * gw.x), -1, 2 * g.nx);
        ky = clampi(__float2int_rd(2.0f * gw.y), -1, 2 * g.ny);
        kz = clampi(__float2int_rd(2.0f * gw.z), -1, 2 * g.nz);
    } else {
        cell_key(g, px, py, pz, kx, ky, kz);
    }
    if (!have || kx != c.kx || ky != c.ky || kz != c.kz) {
        c.kx = kx;
        c.ky = ky;
        c.kz = kz;
        gather_cell(g, pairs, kx, ky, kz, c);
        have = true;
    }
    return interpolate(c, gw);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// x / 6 for the RK4 average: the product with r = RN(1/6) and one residual
// correction by FMA (Markstein's correction step; for a constant divisor see
// Brisebarre and Muller, "Correctly rounded multiplication by arbitrary
// precision constants", 2008).  An exhaustive check over all floats finds it
// equal to the correctly rounded quotient for every |x| >= 2^-120; below
// that the residual underflows and the result may differ in the last place,
// which moves no position (|dt x / 6| is then far below an ulp of any
// coordinate but the smallest).
__device__ __forceinline__ float div6(float x)
{
    const float r = 1.0f / 6.0f;
    const float q = x * r;
    return fmaf(fmaf(-q, 6.0f, x), r, q);
}

// One particle step (psfsolver.cpp:75-224): RK1 or RK4 with the box clamp
// on every stage, lifetime decrement, and respawn from the counter-based
// generator keyed by the caller-order index `perm[idx]` when the lifetime ran
// out (read only then).  `step` is the index of the step being taken (0 for
// the first).
__device__ __forceinline__ float4 advance_particle(float4 p, const GridDev &g, const float2 *__restrict__ u,
                                                   const TraceParams &tp, uint64_t step,
                                                   const int32_t *__restrict__ perm, size_t idx)
{
    if (p.w > 0.f) {
        const float dt = tp.dt;
        CellCache c;
        bool have = false;
        float3 v;
        if (tp.rk4) {
            const float3 k1 = velocity_cached(g, u, p.x, p.y, p.z, c, have);
            float qx = clampf(p.x + 0.5f * dt * k1.x, g.mn[0], g.mx[0]);
            float qy = clampf(p.y + 0.5f * dt * k1.y, g.mn[1], g.mx[1]);
            float qz = clampf(p.z + 0.5f * dt * k1.z, g.mn[2], g.mx[2]);
            const float3 k2 = velocity_cached(g, u, qx, qy, qz, c, have);
            qx = clampf(p.x + 0.5f * dt * k2.x, g.mn[0], g.mx[0]);
            qy = clampf(p.y + 0.5f * dt * k2.y, g.mn[1], g.mx[1]);
            qz = clampf(p.z + 0.5f * dt * k2.z, g.mn[2], g.mx[2]);
            const float3 k3 = velocity_cached(g, u, qx, qy, qz, c, have);
            qx = clampf(p.x + dt * k3.x, g.mn[0], g.mx[0]);
            qy = clampf(p.y + dt * k3.y, g.mn[1], g.mx[1]);
            qz = clampf(p.z + dt * k3.z, g.mn[2], g.mx[2]);
            const float3 k4 = velocity_cached(g, u, qx, qy, qz, c, have);
            v.x = div6(k1.x + 2.f * k2.x + 2.f * k3.x + k4.x);
            v.y = div6(k1.y + 2.f * k2.y + 2.f * k3.y + k4.y);
            v.z = div6(k1.z + 2.f * k2.z + 2.f * k3.z + k4.z);
        } else {
            v = velocity_cached(g, u, p.x, p.y, p.z, c, have);
        }
        p.x = clampf(p.x + dt * v.x, g.mn[0], g.mx[0]);
        p.y = clampf(p.y + dt * v.y, g.mn[1], g.mx[1]);
        p.z = clampf(p.z + dt * v.z, g.mn[2], g.mx[2]);
        p.w = p.w - 1.f;
    } else {
        // psfsolver.cpp:217-222 with the counter-based generator.
        // Particles are stored in cell order; the generator is keyed by the
        // caller's particle index so respawns do not depend on that order.
        const uint32_t id = (uint32_t)perm[idx];
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
