// Mesh voxeliser: the reference's OpenGL slice-map voxelisation
// (Graphics/Model/Model.cpp:203-451, Resources/Voxel/voxel.{vert,geom,frag})
// as three CUDA kernels with no graphics API.
//
//   psf_vox_transform  per vertex: window position in 1/256 pixel and the
//                      crossing height (the reference's projection, Model.cpp:212-213)
//   psf_vox_raster     per triangle: pixel-centre coverage with exact edge
//                      functions; every covered pixel toggles one bit (two in
//                      the layered reference mode) of its voxel column
//   psf_vox_unpack(4)  per column (four columns when the width allows):
//                      suffix parity of the toggles = the XOR of
//                      the reference's prefix masks (voxel.frag:16-52), written
//                      as one inside byte per voxel
//
// The reference XORs the mask "bits [0, n)" of each crossing into the column;
// bit z of the result is the parity of crossings with n > z.  Toggling bit n
// and taking, for each z, the parity of the toggles above z gives the same
// bits with one atomic per covered pixel instead of n/32.
//
// Floating-point steps use explicit round-to-nearest intrinsics in a fixed
// order, so the results match a plain C restatement bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>

#include "psf_internal.h"
#include "psf_voxel.h"

namespace {

constexpr int SUB = 256;            // sub-pixel steps per pixel
constexpr int BIG_PIXELS = 8;       // triangles covering more pixel centres than this are rasterised by a warp
constexpr int RASTER_THREADS = 256;

struct Frame {
    float mn[3], mx[3], ext[3], ctr[3];
    int32_t dims[3];
    int32_t layers;
    int32_t twords;  // toggle words per column
};

struct VoxVert {
    int32_t X, Y;    // window position, 1/256 pixel
    float z;         // reference: slice count from the top; geometric: height in voxels
    float layer;     // reference: slice-map layer
};

// AABB of Model.cpp:73-80 (starts at the origin) and the grid of Model.cpp:205-210.
int frame_of(const psf_voxel_mesh *m, float res, int mode, Frame *f)
{
    using psf::fail;
    if (!m || m->n_vertices < 0 || m->n_triangles < 0) return fail(PSF_ERR_INVALID, "null mesh or negative size");
    if ((m->n_vertices > 0 && !m->vertices) || (m->n_triangles > 0 && !m->triangles))
        return fail(PSF_ERR_INVALID, "null vertex or triangle array");
    if (mode != PSF_VOXEL_REFERENCE && mode != PSF_VOXEL_GEOMETRIC)
        return fail(PSF_ERR_INVALID, "mode must be PSF_VOXEL_REFERENCE or PSF_VOXEL_GEOMETRIC");
    if (!(res > 0.0f) || !std::isfinite(res)) return fail(PSF_ERR_INVALID, "resolution must be positive and finite");
    for (int a = 0; a < 3; ++a) f->mn[a] = f->mx[a] = 0.0f;
    const float *v = m->vertices;
    for (int64_t i = 0; i < m->n_vertices; ++i)
        for (int a = 0; a < 3; ++a) {
            const float p = v[3 * i + a];
            if (!std::isfinite(p)) return fail(PSF_ERR_INVALID, "non-finite vertex coordinate");
            f->mx[a] = std::max(f->mx[a], p);
            f->mn[a] = std::min(f->mn[a], p);
        }
    for (int a = 0; a < 3; ++a) {
        f->ext[a] = f->mx[a] - f->mn[a];
        const float half = 0.5f * f->ext[a];
        f->ctr[a] = f->mn[a] + half;
        const float d = std::ceil(f->ext[a] / res);
        if (!(d >= 1.0f) || d > (float)PSF_VOXEL_MAX_DIM)
            return fail(PSF_ERR_UNSUPPORTED, "the mesh spans no voxel or more than 1023 voxels along an axis");
        f->dims[a] = (int32_t)d;
    }
    f->layers = std::max(1, (int32_t)std::ceil(f->ext[2] / (res * 128.0f)));
    f->twords = mode == PSF_VOXEL_REFERENCE ? 4 * f->layers + 1 : f->dims[2] / 32 + 1;
    return PSF_OK;
}

__global__ void psf_vox_transform(const float *__restrict__ v, int64_t nv, Frame f, float res, int mode,
                                  VoxVert *__restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const float px = v[3 * i], py = v[3 * i + 1], pz = v[3 * i + 2];
    VoxVert o;
    float xw, yw;
    if (mode == PSF_VOXEL_REFERENCE) {
        xw = __fmul_rn(__fdiv_rn(__fsub_rn(px, f.mn[0]), f.ext[0]), (float)f.dims[0]);
        yw = __fmul_rn(__fdiv_rn(__fsub_rn(py, f.mn[1]), f.ext[1]), (float)f.dims[1]);
        const float zo = __fmul_rn(f.ext[2], 0.5f);
        const float top = __fadd_rn(__fsub_rn(f.ctr[2], pz), zo);
        o.z = __fdiv_rn(top, res);
        o.layer = floorf(__fdiv_rn(top, __fmul_rn(res, 128.0f)));
    } else {
        xw = __fdiv_rn(__fsub_rn(px, f.mn[0]), res);
        yw = __fdiv_rn(__fsub_rn(py, f.mn[1]), res);
        o.z = __fdiv_rn(__fsub_rn(pz, f.mn[2]), res);
        o.layer = 0.0f;
    }
    o.X = (int32_t)__float2ll_rn(__fmul_rn(xw, (float)SUB));
    o.Y = (int32_t)__float2ll_rn(__fmul_rn(yw, (float)SUB));
    out[i] = o;
}

// One triangle after setup, in positive orientation A, B, C.
struct Tri {
    int32_t ax, ay, bx, by, cx, cy;
    long long area;
    int32_t own;         // bit 0: edge B->C owns its centres, bit 1: C->A, bit 2: A->B
    int32_t i0, j0, ni;  // first pixel and pixel columns of the bounding box
    int32_t npix;        // pixel centres in the bounding box (0: nothing to draw)
    int32_t lo, n;       // reference mode: toggles at lo (if > 0) and lo + n
    float za, zb, zc;    // geometric mode: crossing heights
};

__device__ __forceinline__ long long edge_fn(long long ax, long long ay, long long bx, long long by, long long px,
                                             long long py)
{
    return (bx - ax) * (py - ay) - (by - ay) * (px - ax);
}

__device__ __forceinline__ int owns(long long dx, long long dy) { return dy < 0 || (dy == 0 && dx > 0); }

__device__ __forceinline__ Tri setup(const VoxVert *__restrict__ q, const uint32_t *__restrict__ tri, int64_t t,
                                     const Frame &f, int mode)
{
    Tri r;
    r.npix = 0;
    const VoxVert v0 = q[tri[3 * t]], v1 = q[tri[3 * t + 1]], v2 = q[tri[3 * t + 2]];
    long long area = edge_fn(v0.X, v0.Y, v1.X, v1.Y, v2.X, v2.Y);
    if (area == 0) return r;
    VoxVert B = v1, C = v2;
    if (area < 0) {
        B = v2;
        C = v1;
        area = -area;
    }
    r.ax = v0.X; r.ay = v0.Y; r.bx = B.X; r.by = B.Y; r.cx = C.X; r.cy = C.Y;
    r.area = area;
    r.own = owns(r.cx - r.bx, r.cy - r.by) | (owns(r.ax - r.cx, r.ay - r.cy) << 1) |
            (owns(r.bx - r.ax, r.by - r.ay) << 2);
    r.za = v0.z; r.zb = B.z; r.zc = C.z;
    r.lo = 0; r.n = 0;
    if (mode == PSF_VOXEL_REFERENCE) {
        // the provoking vertex is the triangle's last one (voxel.geom emits 0, 1, 2)
        const float lay = v2.layer, zc = v2.z;
        if (!(lay >= 0.0f) || lay >= (float)f.layers) return r;
        long long n = zc > 0.0f ? (long long)zc : 0;
        r.n = (int32_t)min(n, 128ll);
        r.lo = 128 * (int32_t)lay;
        if (r.n == 0) return r;
    }
    const int xmin = min(v0.X, min(v1.X, v2.X)), xmax = max(v0.X, max(v1.X, v2.X));
    const int ymin = min(v0.Y, min(v1.Y, v2.Y)), ymax = max(v0.Y, max(v1.Y, v2.Y));
    int i0 = (xmin - SUB / 2 + SUB - 1) / SUB, i1 = xmax < SUB / 2 ? -1 : (xmax - SUB / 2) / SUB;
    int j0 = (ymin - SUB / 2 + SUB - 1) / SUB, j1 = ymax < SUB / 2 ? -1 : (ymax - SUB / 2) / SUB;
    i0 = max(i0, 0); j0 = max(j0, 0);
    i1 = min(i1, f.dims[0] - 1); j1 = min(j1, f.dims[1] - 1);
    if (i1 < i0 || j1 < j0) return r;
    r.i0 = i0; r.j0 = j0; r.ni = i1 - i0 + 1;
    r.npix = r.ni * (j1 - j0 + 1);
    return r;
}

__device__ __forceinline__ void toggle(uint32_t *__restrict__ tog, const Frame &f, int i, int j, int pos)
{
    const size_t hw = (size_t)f.dims[0] * f.dims[1];
    atomicXor(tog + (size_t)(pos >> 5) * hw + (size_t)j * f.dims[0] + i, 1u << (pos & 31));
}

__device__ __forceinline__ void draw(const Tri &r, int p0, int stride, const Frame &f, int mode,
                                     uint32_t *__restrict__ tog)
{
    for (int p = p0; p < r.npix; p += stride) {
        const int i = r.i0 + p % r.ni, j = r.j0 + p / r.ni;
        const long long px = (long long)i * SUB + SUB / 2, py = (long long)j * SUB + SUB / 2;
        const long long e0 = edge_fn(r.bx, r.by, r.cx, r.cy, px, py);
        const long long e1 = edge_fn(r.cx, r.cy, r.ax, r.ay, px, py);
        const long long e2 = edge_fn(r.ax, r.ay, r.bx, r.by, px, py);
        if (!(e0 > 0 || (e0 == 0 && (r.own & 1)))) continue;
        if (!(e1 > 0 || (e1 == 0 && (r.own & 2)))) continue;
        if (!(e2 > 0 || (e2 == 0 && (r.own & 4)))) continue;
        if (mode == PSF_VOXEL_REFERENCE) {
            if (r.lo > 0) toggle(tog, f, i, j, r.lo);
            toggle(tog, f, i, j, r.lo + r.n);
        } else {
            const double s = __dadd_rn(__dadd_rn(__dmul_rn((double)e0, (double)r.za), __dmul_rn((double)e1, (double)r.zb)),
                                       __dmul_rn((double)e2, (double)r.zc));
            const double zc = __ddiv_rn(s, (double)r.area);
            const double t = ceil(__dsub_rn(zc, 0.5));
            const int n = t <= 0.0 ? 0 : (t >= (double)f.dims[2] ? f.dims[2] : (int)t);
            if (n > 0) toggle(tog, f, i, j, n);
        }
    }
}

__device__ __forceinline__ Tri shfl_tri(const Tri &r, int src)
{
    Tri s;
    s.ax = __shfl_sync(0xffffffffu, r.ax, src);
    s.ay = __shfl_sync(0xffffffffu, r.ay, src);
    s.bx = __shfl_sync(0xffffffffu, r.bx, src);
    s.by = __shfl_sync(0xffffffffu, r.by, src);
    s.cx = __shfl_sync(0xffffffffu, r.cx, src);
    s.cy = __shfl_sync(0xffffffffu, r.cy, src);
    s.area = __shfl_sync(0xffffffffu, r.area, src);
    s.own = __shfl_sync(0xffffffffu, r.own, src);
    s.i0 = __shfl_sync(0xffffffffu, r.i0, src);
    s.j0 = __shfl_sync(0xffffffffu, r.j0, src);
    s.ni = __shfl_sync(0xffffffffu, r.ni, src);
    s.npix = __shfl_sync(0xffffffffu, r.npix, src);
    s.lo = __shfl_sync(0xffffffffu, r.lo, src);
    s.n = __shfl_sync(0xffffffffu, r.n, src);
    s.za = __shfl_sync(0xffffffffu, r.za, src);
    s.zb = __shfl_sync(0xffffffffu, r.zb, src);
    s.zc = __shfl_sync(0xffffffffu, r.zc, src);
    return s;
}

// Warp-uniform grid-stride loop over groups of 32 triangles: each lane sets up
// one triangle and draws it alone if it covers few pixel centres; larger ones
// are drawn by the whole warp, one after the other.
__global__ void __launch_bounds__(RASTER_THREADS) psf_vox_raster(const VoxVert *__restrict__ q,
                                                                  const uint32_t *__restrict__ tri, int64_t nt,
                                                                  Frame f, int mode, uint32_t *__restrict__ tog)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < nt; base += nwarps * 32) {
        const int64_t t = base + lane;
        Tri r;
        r.npix = 0;
        if (t < nt) r = setup(q, tri, t, f, mode);
        const bool big = r.npix > BIG_PIXELS;
        if (!big) draw(r, 0, 1, f, mode, tog);
        unsigned m = __ballot_sync(0xffffffffu, big);
        while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            const Tri s = shfl_tri(r, src);
            draw(s, lane, 32, f, mode, tog);
        }
    }
}

// One thread per column: bit z of the column is the parity of the toggles at
// positions above z.
__global__ void psf_vox_unpack(const uint32_t *__restrict__ tog, Frame f, uint8_t *__restrict__ inside)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int W = f.dims[0], H = f.dims[1], D = f.dims[2];
    if (i >= W || j >= H) return;
    const size_t hw = (size_t)W * H, col = (size_t)j * W + i;
    uint32_t carry = 0;  // parity of all toggles in the words above
    for (int w = f.twords - 1; w >= 0; --w) {
        uint32_t x = tog[(size_t)w * hw + col];
        x ^= x >> 1;
        x ^= x >> 2;
        x ^= x >> 4;
        x ^= x >> 8;
        x ^= x >> 16;  // bit k: parity of bits k..31
        const uint32_t above = (x >> 1) ^ (carry ? 0xffffffffu : 0u);
        carry ^= x & 1u;
        const int z0 = 32 * w;
        if (z0 >= D) continue;
        const int zn = min(32, D - z0);
        for (int k = 0; k < zn; ++k) inside[(size_t)(z0 + k) * hw + col] = (uint8_t)((above >> k) & 1u);
    }
}

// The same for grids whose width is a multiple of 4: a thread takes four
// neighbouring columns, reads their toggle words as one 16-byte load and
// writes each z slice of them as one 4-byte store (128 contiguous bytes per
// warp instead of 32).
__device__ __forceinline__ uint32_t suffix_parity(uint32_t x)
{
    x ^= x >> 1;
    x ^= x >> 2;
    x ^= x >> 4;
    x ^= x >> 8;
    x ^= x >> 16;  // bit k: parity of bits k..31
    return x;
}

__global__ void psf_vox_unpack4(const uint32_t *__restrict__ tog, Frame f, uint8_t *__restrict__ inside)
{
    const int i = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int W = f.dims[0], H = f.dims[1], D = f.dims[2];
    if (i >= W || j >= H) return;
    const size_t hw = (size_t)W * H, col = (size_t)j * W + i;
    uint32_t carry = 0;  // bit q: parity of all toggles above, column i + q
    for (int w = f.twords - 1; w >= 0; --w) {
        const uint4 t = *reinterpret_cast<const uint4 *>(tog + (size_t)w * hw + col);
        const uint32_t x0 = suffix_parity(t.x), x1 = suffix_parity(t.y), x2 = suffix_parity(t.z),
                       x3 = suffix_parity(t.w);
        const uint32_t a0 = (x0 >> 1) ^ ((carry & 1u) ? 0xffffffffu : 0u);
        const uint32_t a1 = (x1 >> 1) ^ ((carry & 2u) ? 0xffffffffu : 0u);
        const uint32_t a2 = (x2 >> 1) ^ ((carry & 4u) ? 0xffffffffu : 0u);
        const uint32_t a3 = (x3 >> 1) ^ ((carry & 8u) ? 0xffffffffu : 0u);
        carry ^= (x0 & 1u) | ((x1 & 1u) << 1) | ((x2 & 1u) << 2) | ((x3 & 1u) << 3);
        const int z0 = 32 * w;
        if (z0 >= D) continue;
        const int zn = min(32, D - z0);
        for (int k = 0; k < zn; ++k) {
            const uint32_t v = ((a0 >> k) & 1u) | (((a1 >> k) & 1u) << 8) | (((a2 >> k) & 1u) << 16) |
                               (((a3 >> k) & 1u) << 24);
            *reinterpret_cast<uint32_t *>(inside + (size_t)(z0 + k) * hw + col) = v;
        }
    }
}

}  // namespace

struct psf_voxelizer {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    int64_t max_v = 0, max_t = 0, max_vox = 0;
    float *verts = nullptr;
    uint32_t *tris = nullptr;
    VoxVert *q = nullptr;
    uint8_t *inside = nullptr;
    uint32_t *tog = nullptr;
    size_t tog_words = 0;
    // last run
    bool ready = false;
    Frame f{};
    int mode = 0;
    float res = 0.0f;
    int64_t nv = 0, nt = 0;
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

int launch_all(psf_voxelizer *v)
{
    const Frame &f = v->f;
    const size_t hw = (size_t)f.dims[0] * f.dims[1];
    cudaError_t e = cudaMemsetAsync(v->tog, 0, (size_t)f.twords * hw * sizeof(uint32_t), v->stream);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync");
    if (v->nv > 0) {
        const int64_t blocks = (v->nv + 255) / 256;
        psf_vox_transform<<<(unsigned)blocks, 256, 0, v->stream>>>(v->verts, v->nv, f, v->res, v->mode, v->q);
    }
    if (v->nt > 0) {
        const int64_t need = (v->nt + RASTER_THREADS - 1) / RASTER_THREADS;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)v->sms * 8));
        psf_vox_raster<<<grid, RASTER_THREADS, 0, v->stream>>>(v->q, v->tris, v->nt, f, v->mode, v->tog);
    }
    dim3 blk(32, 8), grd((f.dims[0] + 31) / 32, (f.dims[1] + 7) / 8);
    if (f.dims[0] % 4 == 0) {
        dim3 grd4((f.dims[0] / 4 + 31) / 32, (f.dims[1] + 7) / 8);
        psf_vox_unpack4<<<grd4, blk, 0, v->stream>>>(v->tog, f, v->inside);
    } else {
        psf_vox_unpack<<<grd, blk, 0, v->stream>>>(v->tog, f, v->inside);
    }
    return cuda_status(cudaGetLastError(), "voxeliser launch");
}

}  // namespace

extern "C" {

int psf_voxel_grid(const psf_voxel_mesh *mesh, float resolution, int32_t mode, int32_t dims[3], float aabb[6])
{
    if (!dims || !aabb) return psf::fail(PSF_ERR_INVALID, "null argument");
    Frame f;
    const int rc = frame_of(mesh, resolution, mode, &f);
    if (rc != PSF_OK) return rc;
    for (int a = 0; a < 3; ++a) {
        dims[a] = f.dims[a];
        aabb[a] = f.mn[a];
        aabb[3 + a] = f.mx[a];
    }
    return PSF_OK;
}

int psf_voxelizer_create(int device, int64_t max_vertices, int64_t max_triangles, int64_t max_voxels,
                         psf_voxelizer **out)
{
    if (!out || max_vertices < 1 || max_triangles < 0 || max_voxels < 1)
        return psf::fail(PSF_ERR_INVALID, "null output or non-positive capacity");
    *out = nullptr;
    const cudaError_t es = cudaSetDevice(device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    auto *v = new (std::nothrow) psf_voxelizer();
    if (!v) return psf::fail(PSF_ERR_NOMEM, "host allocation failed");
    v->device = device;
    v->max_v = max_vertices;
    v->max_t = max_triangles;
    v->max_vox = max_voxels;
    cudaDeviceGetAttribute(&v->sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&v->verts, (size_t)max_vertices * 3 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&v->q, (size_t)max_vertices * sizeof(VoxVert));
    if (e == cudaSuccess && max_triangles > 0) e = cudaMalloc(&v->tris, (size_t)max_triangles * 3 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&v->inside, (size_t)max_voxels);
    if (e != cudaSuccess) {
        psf_voxelizer_destroy(v);
        return cuda_status(e, "voxeliser buffers");
    }
    *out = v;
    return PSF_OK;
}

int psf_voxelizer_destroy(psf_voxelizer *v)
{
    if (!v) return psf::fail(PSF_ERR_INVALID, "null voxeliser");
    cudaSetDevice(v->device);
    if (v->stream) cudaStreamSynchronize(v->stream);
    cudaFree(v->verts);
    cudaFree(v->tris);
    cudaFree(v->q);
    cudaFree(v->inside);
    cudaFree(v->tog);
    if (v->stream) cudaStreamDestroy(v->stream);
    delete v;
    return PSF_OK;
}

int psf_voxelizer_run(psf_voxelizer *v, const psf_voxel_mesh *mesh, float resolution, int32_t mode,
                      int32_t dims[3], float aabb[6], uint8_t *inside, int64_t capacity)
{
    if (!v || !dims || !aabb || !inside) return psf::fail(PSF_ERR_INVALID, "null argument");
    Frame f;
    int rc = frame_of(mesh, resolution, mode, &f);
    if (rc != PSF_OK) return rc;
    for (int a = 0; a < 3; ++a) {
        dims[a] = f.dims[a];
        aabb[a] = f.mn[a];
        aabb[3 + a] = f.mx[a];
    }
    const int64_t nvox = (int64_t)f.dims[0] * f.dims[1] * f.dims[2];
    if (capacity < nvox) return psf::fail(PSF_ERR_INVALID, "output smaller than the voxel grid");
    if (mesh->n_vertices > v->max_v || mesh->n_triangles > v->max_t || nvox > v->max_vox)
        return psf::fail(PSF_ERR_INVALID, "mesh or grid larger than the voxeliser was created for");
    const uint32_t *t = mesh->triangles;
    for (int64_t i = 0; i < 3 * mesh->n_triangles; ++i)
        if ((int64_t)t[i] >= mesh->n_vertices) return psf::fail(PSF_ERR_INVALID, "triangle index out of range");
    const cudaError_t es = cudaSetDevice(v->device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    const size_t hw = (size_t)f.dims[0] * f.dims[1];
    const size_t words = (size_t)f.twords * hw;
    if (words > v->tog_words) {
        cudaStreamSynchronize(v->stream);
        cudaFree(v->tog);
        v->tog = nullptr;
        v->tog_words = 0;
        const cudaError_t e = cudaMalloc(&v->tog, words * sizeof(uint32_t));
        if (e != cudaSuccess) return cuda_status(e, "cudaMalloc");
        v->tog_words = words;
    }
    v->ready = false;
    v->f = f;
    v->mode = mode;
    v->res = resolution;
    v->nv = mesh->n_vertices;
    v->nt = mesh->n_triangles;
    cudaError_t e = cudaSuccess;
    if (v->nv > 0)
        e = cudaMemcpyAsync(v->verts, mesh->vertices, (size_t)v->nv * 3 * sizeof(float), cudaMemcpyHostToDevice,
                            v->stream);
    if (e == cudaSuccess && v->nt > 0)
        e = cudaMemcpyAsync(v->tris, mesh->triangles, (size_t)v->nt * 3 * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            v->stream);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemcpyAsync");
    rc = launch_all(v);
    if (rc != PSF_OK) return rc;
    e = cudaMemcpyAsync(inside, v->inside, (size_t)nvox, cudaMemcpyDeviceToHost, v->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v->stream);
    if (e != cudaSuccess) return cuda_status(e, "voxeliser read-back");
    v->ready = true;
    return PSF_OK;
}

int psf_voxelizer_profile(psf_voxelizer *v, int32_t iters, double *ms)
{
    if (!v || !ms || iters < 1) return psf::fail(PSF_ERR_INVALID, "null argument or iters < 1");
    if (!v->ready) return psf::fail(PSF_ERR_STATE, "no voxelisation has run yet");
    const cudaError_t es = cudaSetDevice(v->device);
    if (es != cudaSuccess) return psf::cuda_fail(es, "cudaSetDevice");
    cudaEvent_t a, b;
    cudaError_t ec = cudaEventCreate(&a);
    if (ec != cudaSuccess) return psf::cuda_fail(ec, "cudaEventCreate");
    ec = cudaEventCreate(&b);
    if (ec != cudaSuccess) {
        cudaEventDestroy(a);
        return psf::cuda_fail(ec, "cudaEventCreate");
    }
    int rc = launch_all(v);  // warm-up
    cudaEventRecord(a, v->stream);
    for (int k = 0; k < iters && rc == PSF_OK; ++k) rc = launch_all(v);
    cudaEventRecord(b, v->stream);
    const cudaError_t e = cudaEventSynchronize(b);
    float t = 0.0f;
    if (rc == PSF_OK && e == cudaSuccess) {
        cudaEventElapsedTime(&t, a, b);
        *ms = (double)t / iters;
    } else if (rc == PSF_OK) {
        rc = psf::cuda_fail(e, "cudaEventSynchronize");
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

int psf_voxelize(const psf_voxel_mesh *mesh, float resolution, int32_t mode, int device, int32_t dims[3],
                 float aabb[6], uint8_t *inside, int64_t capacity)
{
    if (!mesh || !dims || !aabb || !inside) return psf::fail(PSF_ERR_INVALID, "null argument");
    int rc = psf_voxel_grid(mesh, resolution, mode, dims, aabb);
    if (rc != PSF_OK) return rc;
    const int64_t nvox = (int64_t)dims[0] * dims[1] * dims[2];
    if (capacity < nvox) return psf::fail(PSF_ERR_INVALID, "output smaller than the voxel grid");
    psf_voxelizer *v = nullptr;
    rc = psf_voxelizer_create(device, std::max<int64_t>(1, mesh->n_vertices), mesh->n_triangles, nvox, &v);
    if (rc != PSF_OK) return rc;
    rc = psf_voxelizer_run(v, mesh, resolution, mode, dims, aabb, inside, capacity);
    psf_voxelizer_destroy(v);
    return rc;
}

}  // extern "C"
