// Particle density volume and its ray-marched image: the compute part of the
// reference's PSFSolverGPU::drawParticles (Solver/SolverImpl/psfsolvergpu.cpp:876-1022)
// as CUDA kernels writing device buffers, with no graphics API.
//
//   psf_vol_histogram  particle -> cell counts; a warp merges equal cells
//                      (__match_any_sync) before one atomic per distinct cell
//   psf_vol_density    counts / 1e6 -> FP16 density, and clears the counts for
//                      the next frame (volume.comp, Texture3D::clearImage)
//   psf_vol_render     one thread per pixel: ray/AABB slab test, march with
//                      trilinear clamp-to-border samples, shadow ray toward the
//                      light, front-to-back emission/absorption (volume.frag)
//
// The density (R^3 FP16, 32 MB at R = 256) stays L2-resident while a frame is
// rendered.  Arithmetic is round-to-nearest FP32 through explicit intrinsics
// in a fixed order (no contraction), so results equal a plain C restatement
// bit for bit.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>

#include "psf_internal.h"
#include "psf_volume.h"

namespace {

constexpr float VOL_ZDIR = -1.792590986919304f;          // -1 / tan(45.0 / 2.0), radians as in volume.frag
constexpr float VOL_SHADOW_THRESH = 6.907755278982137f;  // -log(0.001) / 1.0

struct Box {
    float mn[3], mx[3], ext[3];
    int R;
};

struct View {
    float view[16];
    float cam[3], light[3];
    float mn[3], mx[3];
    int W, H, R;
};

// Grid-stride over groups of 32 particles so every lane takes part in the match.
__global__ void psf_vol_histogram(const float4 *__restrict__ p, long long n, Box b, int *__restrict__ hist)
{
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * 32; base < n; base += nwarps * 32) {
        const long long i = base + lane;
        long long key = -1;
        if (i < n) {
            const float4 q = p[i];
            const float c[3] = {q.x, q.y, q.z};
            long long idx = 0;
            bool ok = true;
            for (int a = 2; a >= 0; --a) {
                const float t = __fdiv_rn(__fsub_rn(c[a], b.mn[a]), b.ext[a]);
                const float f = floorf(__fmul_rn(t, (float)b.R));
                if (!(f >= 0.0f) || f >= (float)b.R) ok = false;
                else idx = idx * b.R + (long long)f;
            }
            if (ok) key = idx;
        }
        const unsigned same = __match_any_sync(0xffffffffu, key);
        if (key >= 0 && lane == __ffs(same) - 1) atomicAdd(hist + key, __popc(same));
    }
}

__global__ void psf_vol_density(int *__restrict__ hist, __half *__restrict__ vol, long long cells)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += stride) {
        const int h = hist[i];
        vol[i] = __float2half_rn(__fdiv_rn((float)h, 1000000.0f));
        hist[i] = 0;
    }
}

__device__ __forceinline__ float texel(const __half *__restrict__ v, int R, int x, int y, int z)
{
    if (x < 0 || y < 0 || z < 0 || x >= R || y >= R || z >= R) return 0.0f;
    return __half2float(v[((long long)z * R + y) * R + x]);
}

__device__ __forceinline__ float lerp1(float a, float b, float t)
{
    return __fadd_rn(__fmul_rn(__fsub_rn(1.0f, t), a), __fmul_rn(t, b));
}

__device__ float sample(const __half *__restrict__ v, int R, float px, float py, float pz)
{
    const float u = __fsub_rn(__fmul_rn(px, (float)R), 0.5f);
    const float w1 = __fsub_rn(__fmul_rn(py, (float)R), 0.5f);
    const float w2 = __fsub_rn(__fmul_rn(pz, (float)R), 0.5f);
    const float fu = floorf(u), fv = floorf(w1), fw = floorf(w2);
    if (!(fu >= -1.0f && fu < (float)R && fv >= -1.0f && fv < (float)R && fw >= -1.0f && fw < (float)R))
        return 0.0f;
    const float a = __fsub_rn(u, fu), b = __fsub_rn(w1, fv), c = __fsub_rn(w2, fw);
    const int x = (int)fu, y = (int)fv, z = (int)fw;
    const float c00 = lerp1(texel(v, R, x, y, z), texel(v, R, x + 1, y, z), a);
    const float c10 = lerp1(texel(v, R, x, y + 1, z), texel(v, R, x + 1, y + 1, z), a);
    const float c01 = lerp1(texel(v, R, x, y, z + 1), texel(v, R, x + 1, y, z + 1), a);
    const float c11 = lerp1(texel(v, R, x, y + 1, z + 1), texel(v, R, x + 1, y + 1, z + 1), a);
    const float c0 = lerp1(c00, c10, b), c1 = lerp1(c01, c11, b);
    return lerp1(c0, c1, c);
}

// exp(-y) for y in [0, 1]: Taylor series to degree 12, Horner form.
__device__ __forceinline__ float exp_neg_unit(float y)
{
    const float x = -y;
    float r = 1.0f;
#pragma unroll
    for (int k = 12; k >= 1; --k) r = __fadd_rn(1.0f, __fmul_rn(__fdiv_rn(x, (float)k), r));
    return r;
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ float len3(float x, float y, float z)
{
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}

__global__ void __launch_bounds__(256) psf_vol_render(const __half *__restrict__ vol, View V, float4 *__restrict__ out)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= V.W || py >= V.H) return;
    const int R = V.R;
    float ext[3];
    for (int a = 0; a < 3; ++a) ext[a] = __fsub_rn(V.mx[a], V.mn[a]);
    const float vox = __fmul_rn(__fmul_rn(__fdiv_rn(ext[0], (float)R), __fdiv_rn(ext[1], (float)R)),
                                __fdiv_rn(ext[2], (float)R));
    const float step = __fdiv_rn(ext[0], 256.0f);
    float lview[3];
    for (int i = 0; i < 3; ++i)
        lview[i] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(V.view[i], V.light[0]), __fmul_rn(V.view[4 + i], V.light[1])),
                                       __fmul_rn(V.view[8 + i], V.light[2])),
                             __fmul_rn(V.view[12 + i], 1.0f));
    float r0 = __fsub_rn(__fdiv_rn(__fmul_rn(2.0f, __fadd_rn((float)px, 0.5f)), (float)V.W), 1.0f);
    const float r1 = __fsub_rn(__fdiv_rn(__fmul_rn(2.0f, __fadd_rn((float)py, 0.5f)), (float)V.H), 1.0f);
    r0 = __fmul_rn(r0, __fdiv_rn((float)V.W, (float)V.H));
    const float r2 = VOL_ZDIR;
    float d[3];
    for (int j = 0; j < 3; ++j) {
        const float *col = V.view + 4 * j;
        d[j] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r0, col[0]), __fmul_rn(r1, col[1])), __fmul_rn(r2, col[2])),
                         __fmul_rn(0.0f, col[3]));
    }
    float tmin[3], tmax[3];
    for (int a = 0; a < 3; ++a) {
        const float inv = __fdiv_rn(1.0f, d[a]);
        const float tt = __fmul_rn(inv, __fsub_rn(V.mx[a], V.cam[a]));
        const float tb = __fmul_rn(inv, __fsub_rn(V.mn[a], V.cam[a]));
        tmin[a] = fminf(tt, tb);
        tmax[a] = fmaxf(tt, tb);
    }
    const float t0 = fmaxf(0.0f, fmaxf(fmaxf(tmin[0], tmin[1]), fmaxf(tmin[0], tmin[2])));
    const float t1 = fminf(fminf(tmax[0], tmax[1]), fminf(tmax[0], tmax[2]));
    float pos[3], ray[3];
    for (int a = 0; a < 3; ++a) {
        const float s0 = __fdiv_rn(__fsub_rn(__fadd_rn(V.cam[a], __fmul_rn(d[a], t0)), V.mn[a]), ext[a]);
        const float s1 = __fdiv_rn(__fsub_rn(__fadd_rn(V.cam[a], __fmul_rn(d[a], t1)), V.mn[a]), ext[a]);
        pos[a] = s0;
        ray[a] = __fsub_rn(s1, s0);
    }
    float rl = len3(ray[0], ray[1], ray[2]);
    float sv[3];
    for (int a = 0; a < 3; ++a) sv[a] = __fdiv_rn(__fmul_rn(step, ray[a]), rl);
    float trans = 1.0f, le0 = 0.0f, le1 = 0.0f, le2 = 0.0f;
    int steps = 1024;
    while (rl > 0.0f && steps > 0) {
        const float s = __fdiv_rn(sample(vol, R, pos[0], pos[1], pos[2]), vox);
        if (s > 0.001f) {
            const float lx = __fsub_rn(lview[0], pos[0]), ly = __fsub_rn(lview[1], pos[1]),
                        lz = __fsub_rn(lview[2], pos[2]);
            const float ll = len3(lx, ly, lz);
            const float lv0 = __fdiv_rn(__fmul_rn(step, lx), ll), lv1 = __fdiv_rn(__fmul_rn(step, ly), ll),
                        lv2 = __fdiv_rn(__fmul_rn(step, lz), ll);
            float l0 = pos[0], l1 = pos[1], l2 = pos[2];
            float sd = 0.0f;
            for (int i = 0; i < 128; ++i) {
                l0 = __fadd_rn(l0, lv0);
                l1 = __fadd_rn(l1, lv1);
                l2 = __fadd_rn(l2, lv2);
                sd = __fadd_rn(sd, __fdiv_rn(sample(vol, R, l0, l1, l2), vox));
                if (sd > VOL_SHADOW_THRESH) break;
            }
            const float dens = clampf(__fmul_rn(s, step), 0.0f, 1.0f);
            const float e = exp_neg_unit(clampf(__fmul_rn(sd, step), 0.0f, 1.0f));
            const float sh0 = __fmul_rn(1.0f, e), sh1 = __fmul_rn(0.5f, e), sh2 = __fmul_rn(0.0f, e);
            le0 = __fadd_rn(le0, __fmul_rn(__fmul_rn(sh0, dens), trans));
            le1 = __fadd_rn(le1, __fmul_rn(__fmul_rn(sh1, dens), trans));
            le2 = __fadd_rn(le2, __fmul_rn(__fmul_rn(sh2, dens), trans));
            trans = __fmul_rn(trans, __fsub_rn(1.0f, dens));
            if (trans < 0.01f) break;
            le0 = clampf(le0, 0.0f, 1.0f);
            le1 = clampf(le1, 0.0f, 1.0f);
            le2 = clampf(le2, 0.0f, 1.0f);
            trans = clampf(trans, 0.0f, 1.0f);
        }
        rl = __fsub_rn(rl, step);
        for (int a = 0; a < 3; ++a) pos[a] = __fadd_rn(pos[a], sv[a]);
        --steps;
    }
    out[(long long)py * V.W + px] = make_float4(le0, le1, le2, trans);
}

}  // namespace

struct psf_volume {
    int device = 0;
    int sms = 148;
    int R = 256;
    cudaStream_t stream = nullptr;  // own stream (host splats and renders)
    int *hist = nullptr;
    __half *vol = nullptr;
    float4 *parts = nullptr;        // host-splat staging
    long long parts_cap = 0;
    float4 *img = nullptr;
    long long img_cap = 0;
    // last host splat (its particles stay in `parts`), for profiling
    const float4 *last_parts = nullptr;
    long long last_n = -1;
    Box last_box{};
    bool have_density = false;
};

namespace {

int cuda_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return PSF_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return psf::fail(PSF_ERR_NOMEM, std::string(what) + ": out of device memory");
    }
    return psf::cuda_fail(e, what);
}

int make_box(const float *mn, const float *mx, int R, Box *b)
{
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(mn[a]) || !std::isfinite(mx[a]) || !(mx[a] > mn[a]))
            return psf::fail(PSF_ERR_INVALID, "the box must have max > min on every axis");
        b->mn[a] = mn[a];
        b->mx[a] = mx[a];
        b->ext[a] = mx[a] - mn[a];
    }
    b->R = R;
    return PSF_OK;
}

int launch_splat(psf_volume *v, const float4 *parts, long long n, const Box &b, cudaStream_t st)
{
    const long long cells = (long long)v->R * v->R * v->R;
    if (n > 0) {
        const long long need = (n + 255) / 256;
        const int grid = (int)std::max<long long>(1, std::min<long long>(need, (long long)v->sms * 8));
        psf_vol_histogram<<<grid, 256, 0, st>>>(parts, n, b, v->hist);
    }
    const int grid = (int)std::min<long long>((cells + 255) / 256, (long long)v->sms * 16);
    psf_vol_density<<<grid, 256, 0, st>>>(v->hist, v->vol, cells);
    return cuda_status(cudaGetLastError(), "volume splat launch");
}

int check_view(const psf_volume_view *view)
{
    if (!view) return psf::fail(PSF_ERR_INVALID, "null view");
    if (view->width < 1 || view->height < 1 || (long long)view->width * view->height > (1ll << 28))
        return psf::fail(PSF_ERR_INVALID, "image size must be positive and at most 2^28 pixels");
    return PSF_OK;
}

int launch_render(psf_volume *v, const psf_volume_view *view, cudaStream_t st)
{
    View V;
    std::memcpy(V.view, view->view, sizeof(V.view));
    for (int a = 0; a < 3; ++a) {
        V.cam[a] = view->camera[a];
        V.light[a] = view->light[a];
        V.mn[a] = v->last_box.mn[a];
        V.mx[a] = v->last_box.mx[a];
    }
    V.W = view->width;
    V.H = view->height;
    V.R = v->R;
    dim3 blk(16, 16), grd((V.W + 15) / 16, (V.H + 15) / 16);
    psf_vol_render<<<grd, blk, 0, st>>>(v->vol, V, v->img);
    return cuda_status(cudaGetLastError(), "volume render launch");
}

int ensure_image(psf_volume *v, long long pixels)
{
    if (pixels <= v->img_cap) return PSF_OK;
    cudaStreamSynchronize(v->stream);
    cudaFree(v->img);
    v->img = nullptr;
    v->img_cap = 0;
    const cudaError_t e = cudaMalloc(&v->img, (size_t)pixels * sizeof(float4));
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc");
    v->img_cap = pixels;
    return PSF_OK;
}

}  // namespace

extern "C" {

int psf_volume_create(int device, int32_t res, psf_volume **out)
{
    if (!out) return psf::fail(PSF_ERR_INVALID, "null output");
    *out = nullptr;
    if (res < 2 || res > PSF_VOLUME_MAX_RES) return psf::fail(PSF_ERR_UNSUPPORTED, "res must be in [2, 512]");
    const cudaError_t es = cudaSetDevice(device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    auto *v = new (std::nothrow) psf_volume();
    if (!v) return psf::fail(PSF_ERR_NOMEM, "host allocation failed");
    v->device = device;
    v->R = res;
    cudaDeviceGetAttribute(&v->sms, cudaDevAttrMultiProcessorCount, device);
    const size_t cells = (size_t)res * res * res;
    cudaError_t e = cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&v->hist, cells * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&v->vol, cells * sizeof(__half));
    if (e == cudaSuccess) e = cudaMemsetAsync(v->hist, 0, cells * sizeof(int), v->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(v->vol, 0, cells * sizeof(__half), v->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
    if (e != cudaSuccess) {
        psf_volume_destroy(v);
        return cuda_status(e, "volume buffers");
    }
    *out = v;
    return PSF_OK;
}

int psf_volume_destroy(psf_volume *v)
{
    if (!v) return psf::fail(PSF_ERR_INVALID, "null volume");
    cudaSetDevice(v->device);
    if (v->stream) cudaStreamSynchronize(v->stream);
    cudaFree(v->hist);
    cudaFree(v->vol);
    cudaFree(v->parts);
    cudaFree(v->img);
    if (v->stream) cudaStreamDestroy(v->stream);
    delete v;
    return PSF_OK;
}

int psf_volume_splat(psf_volume *v, const float *particles, int64_t n, const float aabb_min[3],
                     const float aabb_max[3])
{
    if (!v || !aabb_min || !aabb_max || n < 0 || (n > 0 && !particles))
        return psf::fail(PSF_ERR_INVALID, "null argument or negative count");
    Box b;
    int rc = make_box(aabb_min, aabb_max, v->R, &b);
    if (rc != PSF_OK) return rc;
    const cudaError_t es = cudaSetDevice(v->device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    if (n > v->parts_cap) {
        cudaStreamSynchronize(v->stream);
        cudaFree(v->parts);
        v->parts = nullptr;
        v->parts_cap = 0;
        const cudaError_t e = cudaMalloc(&v->parts, (size_t)n * sizeof(float4));
        if (e != cudaSuccess) return cuda_status(e, "cudaMalloc");
        v->parts_cap = n;
    }
    if (n > 0) {
        const cudaError_t e = cudaMemcpyAsync(v->parts, particles, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice,
                                              v->stream);
        if (e != cudaSuccess) return cuda_status(e, "cudaMemcpyAsync");
    }
    rc = launch_splat(v, v->parts, n, b, v->stream);
    if (rc != PSF_OK) return rc;
    const cudaError_t e = cudaStreamSynchronize(v->stream);
    if (e != cudaSuccess) return cuda_status(e, "volume splat");
    v->last_parts = v->parts;
    v->last_n = n;
    v->last_box = b;
    v->have_density = true;
    return PSF_OK;
}

int psf_volume_splat_context(psf_volume *v, psf_ctx *ctx)
{
    if (!v || !ctx) return psf::fail(PSF_ERR_INVALID, "null argument");
    psf::ContextParticles cp;
    int rc = psf::context_particles(ctx, &cp);
    if (rc != PSF_OK) return rc;
    if (cp.device != v->device) return psf::fail(PSF_ERR_INVALID, "the context lives on another device");
    if (cp.n > 0 && !cp.parts) return psf::fail(PSF_ERR_STATE, "the context has no particles");
    Box b;
    rc = make_box(cp.mn, cp.mx, v->R, &b);
    if (rc != PSF_OK) return rc;
    const cudaError_t es = cudaSetDevice(v->device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    // Runs on the context's stream, after its queued steps.
    rc = launch_splat(v, cp.parts, cp.n, b, cp.stream);
    if (rc != PSF_OK) return rc;
    const cudaError_t e = cudaStreamSynchronize(cp.stream);
    if (e != cudaSuccess) return cuda_status(e, "volume splat");
    // The context owns its particles; profiling needs a host splat.
    v->last_parts = nullptr;
    v->last_n = -1;
    v->last_box = b;
    v->have_density = true;
    return PSF_OK;
}

int psf_volume_get_density(psf_volume *v, uint16_t *density, int64_t count)
{
    if (!v || !density) return psf::fail(PSF_ERR_INVALID, "null argument");
    const long long cells = (long long)v->R * v->R * v->R;
    if (count < cells) return psf::fail(PSF_ERR_INVALID, "output smaller than res^3");
    const cudaError_t es = cudaSetDevice(v->device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    cudaError_t e = cudaMemcpyAsync(density, v->vol, (size_t)cells * sizeof(__half), cudaMemcpyDeviceToHost, v->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
    return cuda_status(e, "density read-back");
}

int psf_volume_render(psf_volume *v, const psf_volume_view *view, float *rgba, int64_t count)
{
    if (!v || !rgba) return psf::fail(PSF_ERR_INVALID, "null argument");
    int rc = check_view(view);
    if (rc != PSF_OK) return rc;
    if (!v->have_density) return psf::fail(PSF_ERR_STATE, "no density yet: splat particles first");
    const long long pixels = (long long)view->width * view->height;
    if (count < 4 * pixels) return psf::fail(PSF_ERR_INVALID, "output smaller than width * height * 4");
    const cudaError_t es = cudaSetDevice(v->device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    if ((rc = ensure_image(v, pixels)) != PSF_OK) return rc;
    if ((rc = launch_render(v, view, v->stream)) != PSF_OK) return rc;
    cudaError_t e = cudaMemcpyAsync(rgba, v->img, (size_t)pixels * sizeof(float4), cudaMemcpyDeviceToHost, v->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
    return cuda_status(e, "image read-back");
}

int psf_volume_profile(psf_volume *v, const psf_volume_view *view, int32_t iters, double *splat_ms,
                       double *render_ms)
{
    if (!v || !splat_ms || !render_ms || iters < 1) return psf::fail(PSF_ERR_INVALID, "null argument or iters < 1");
    int rc = check_view(view);
    if (rc != PSF_OK) return rc;
    if (!v->have_density || v->last_n < 0)
        return psf::fail(PSF_ERR_STATE, "profiling re-splats the particles of the last psf_volume_splat");
    const cudaError_t es = cudaSetDevice(v->device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    if ((rc = ensure_image(v, (long long)view->width * view->height)) != PSF_OK) return rc;
    cudaEvent_t ev[3];
    for (int i = 0; i < 3; ++i) {
        const cudaError_t e = cudaEventCreate(&ev[i]);
        if (e != cudaSuccess) {
            for (int k = 0; k < i; ++k) cudaEventDestroy(ev[k]);
            return psf::cuda_fail(e, "cudaEventCreate");
        }
    }
    cudaStream_t st = v->stream;
    rc = launch_splat(v, v->last_parts, v->last_n, v->last_box, st);  // warm-up
    if (rc == PSF_OK) rc = launch_render(v, view, st);
    cudaEventRecord(ev[0], st);
    for (int k = 0; k < iters && rc == PSF_OK; ++k) rc = launch_splat(v, v->last_parts, v->last_n, v->last_box, st);
    cudaEventRecord(ev[1], st);
    for (int k = 0; k < iters && rc == PSF_OK; ++k) rc = launch_render(v, view, st);
    cudaEventRecord(ev[2], st);
    const cudaError_t e = cudaEventSynchronize(ev[2]);
    if (rc == PSF_OK && e != cudaSuccess) rc = psf::cuda_fail(e, "cudaEventSynchronize");
    if (rc == PSF_OK) {
        float a = 0.0f, b = 0.0f;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        *splat_ms = (double)a / iters;
        *render_ms = (double)b / iters;
    }
    for (int i = 0; i < 3; ++i) cudaEventDestroy(ev[i]);
    return rc;
}

}  // extern "C"
