/*
 * Test infrastructure (oracle): CPU restatement of the reference's mesh
 * voxeliser, used only by tests/ and by bench.py's CPU baseline leg.
 *
 * The reference turns a closed triangle mesh into the simulation domain with
 * a "slice map" drawn by OpenGL (Graphics/Model/Model.cpp:203-451 with
 * Resources/Voxel/voxel.vert, voxel.geom, voxel.frag):
 *
 *   - the model's AABB starts at the origin and grows over every vertex
 *     (Graphics/Model/Model.cpp:73-80, Graphics/AABB/AABB.cpp:3-7);
 *   - width/height/depth = ceil(extent / resolution), layers =
 *     ceil(extent.z / (resolution * 128)) (Model.cpp:205-210);
 *   - the mesh is drawn with an orthographic xy projection onto a
 *     width x height viewport (Model.cpp:212-213, 247), every triangle
 *     rasterised at pixel centres, culling and depth test off, and XOR as
 *     the colour logic op (Model.cpp:249-256);
 *   - each fragment writes a 128-bit mask (RGBA32UI) with bits [0, z) set,
 *     where z = uint((pos.z + extent.z/2) / resolution) and pos is the
 *     provoking vertex's projected position (flat input; the projection
 *     negates z, so z counts down from the top of the box), into the layer
 *     floor((pos.z + extent.z/2) / (128 * resolution)) of the provoking
 *     vertex (voxel.geom:14-22, voxel.frag:16-52);
 *   - after drawing, bit d of channel c of layer l marks voxel
 *     (x, y, 128 l + 32 c + d) inside (Model.cpp:278-441).
 *
 * XOR-accumulating prefix masks leaves bit d set where an odd number of
 * surface crossings lies above it, i.e. inside a closed surface.
 *
 * GL's rasteriser is implementation-defined in its sub-pixel precision and
 * in how it breaks ties on shared edges; both are fixed here: vertices snap
 * to 1/256 pixel, coverage is tested with exact 64-bit edge functions at
 * pixel centres, and an edge owns the centres on it when, walked in the
 * positive orientation, it goes down (dy < 0) or is horizontal going right.
 * The CUDA voxeliser uses exactly these rules and the same floating-point
 * operations (no contraction: this file is built with -ffp-contract=off),
 * so the two agree bit for bit.
 *
 * Mode 1 ("geometric") is this project's corrected variant: pixels and voxel
 * columns coincide (pixel size = resolution), the crossing height is the
 * triangle's plane interpolated at the pixel centre, voxel z counts up from
 * the bottom, and voxel (x, y, z) is inside when an odd number of crossings
 * lies above its centre.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define VOX_SUB 256      /* sub-pixel steps per pixel */
#define VOX_MAX_DIM 1023 /* voxels per axis */

typedef struct {
    float mn[3], mx[3], ext[3], ctr[3];
    int32_t dims[3];
    int32_t layers;
    int32_t words; /* 32-bit words per column */
} vox_frame;

/* AABB and grid of the reference's voxelize (Model.cpp:73-80, 205-210). */
static int vox_frame_of(const float *v, int64_t nv, float res, int mode, vox_frame *f)
{
    if (!(res > 0.0f) || !isfinite(res)) return -1;
    for (int a = 0; a < 3; ++a) f->mn[a] = f->mx[a] = 0.0f;
    for (int64_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a) {
            float p = v[3 * i + a];
            if (!isfinite(p)) return -1;
            if (p > f->mx[a]) f->mx[a] = p;
            if (p < f->mn[a]) f->mn[a] = p;
        }
    for (int a = 0; a < 3; ++a) {
        f->ext[a] = f->mx[a] - f->mn[a];
        f->ctr[a] = f->mn[a] + 0.5f * (f->mx[a] - f->mn[a]);
        float d = ceilf(f->ext[a] / res);
        if (!(d >= 1.0f) || d > (float)VOX_MAX_DIM) return -1;
        f->dims[a] = (int32_t)d;
    }
    f->layers = (int32_t)ceilf(f->ext[2] / (res * 128.0f));
    if (f->layers < 1) f->layers = 1;
    f->words = mode == 0 ? 4 * f->layers : (f->dims[2] + 31) / 32;
    return 0;
}

typedef struct {
    int64_t X, Y;  /* window position in 1/256 pixel */
    float z;       /* mode 0: slice count from the top; mode 1: height in voxels from the bottom */
    float layer;   /* mode 0: slice-map layer */
} vox_vert;

static vox_vert vox_transform(const vox_frame *f, const float *p, float res, int mode)
{
    vox_vert o;
    float xw, yw;
    if (mode == 0) {
        xw = (p[0] - f->mn[0]) / f->ext[0] * (float)f->dims[0];
        yw = (p[1] - f->mn[1]) / f->ext[1] * (float)f->dims[1];
        float zo = f->ext[2] * 0.5f;
        float top = (f->ctr[2] - p[2]) + zo;
        o.z = top / res;
        o.layer = floorf(top / (res * 128.0f));
    } else {
        xw = (p[0] - f->mn[0]) / res;
        yw = (p[1] - f->mn[1]) / res;
        o.z = (p[2] - f->mn[2]) / res;
        o.layer = 0.0f;
    }
    o.X = (int64_t)rintf(xw * (float)VOX_SUB);
    o.Y = (int64_t)rintf(yw * (float)VOX_SUB);
    return o;
}

static int64_t edge_fn(int64_t ax, int64_t ay, int64_t bx, int64_t by, int64_t px, int64_t py)
{
    return (bx - ax) * (py - ay) - (by - ay) * (px - ax);
}

static int owns(int64_t dx, int64_t dy) { return dy < 0 || (dy == 0 && dx > 0); }

static void xor_range(uint32_t *col, int64_t lo, int64_t hi)
{
    for (int64_t b = lo; b < hi;) {
        int64_t w = b >> 5;
        int64_t end = (w + 1) << 5;
        if (end > hi) end = hi;
        int s = (int)(b & 31), n = (int)(end - b);
        uint32_t m = n == 32 ? 0xFFFFFFFFu : (((1u << n) - 1u) << s);
        col[w] ^= m;
        b = end;
    }
}

/* Grid of a mesh: dims[3] and aabb[6] = (min, max).  0, or -1 for an empty,
 * flat, non-finite or too-large mesh. */
int psfo_voxel_dims(const float *v, int64_t nv, float res, int mode, int32_t *dims, float *aabb)
{
    vox_frame f;
    if (vox_frame_of(v, nv, res, mode, &f)) return -1;
    for (int a = 0; a < 3; ++a) {
        dims[a] = f.dims[a];
        aabb[a] = f.mn[a];
        aabb[3 + a] = f.mx[a];
    }
    return 0;
}

/* Inside flags [depth][height][width] (1 = inside).  -1 on a bad mesh or a
 * triangle index out of range. */
int psfo_voxelize(const float *v, int64_t nv, const uint32_t *tri, int64_t nt, float res, int mode, uint8_t *inside)
{
    vox_frame f;
    if (vox_frame_of(v, nv, res, mode, &f)) return -1;
    const int W = f.dims[0], H = f.dims[1], D = f.dims[2];
    uint32_t *cols = (uint32_t *)calloc((size_t)W * H * f.words, sizeof(uint32_t));
    if (!cols) return -1;
    for (int64_t t = 0; t < nt; ++t) {
        uint32_t id[3] = {tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]};
        if (id[0] >= nv || id[1] >= nv || id[2] >= nv) {
            free(cols);
            return -1;
        }
        vox_vert q[3];
        for (int k = 0; k < 3; ++k) q[k] = vox_transform(&f, v + 3 * (int64_t)id[k], res, mode);
        int64_t area = edge_fn(q[0].X, q[0].Y, q[1].X, q[1].Y, q[2].X, q[2].Y);
        if (area == 0) continue;
        /* positive orientation: a = 0, b = 1, c = 2 or a = 0, b = 2, c = 1 */
        int b = 1, c = 2;
        if (area < 0) {
            b = 2;
            c = 1;
            area = -area;
        }
        const vox_vert *A = &q[0], *B = &q[b], *C = &q[c];
        int64_t xmin = A->X, xmax = A->X, ymin = A->Y, ymax = A->Y;
        for (int k = 1; k < 3; ++k) {
            if (q[k].X < xmin) xmin = q[k].X;
            if (q[k].X > xmax) xmax = q[k].X;
            if (q[k].Y < ymin) ymin = q[k].Y;
            if (q[k].Y > ymax) ymax = q[k].Y;
        }
        /* pixel centres (i + 1/2) inside [min, max] */
        int64_t i0 = (xmin - VOX_SUB / 2 + VOX_SUB - 1) / VOX_SUB, i1 = (xmax - VOX_SUB / 2) / VOX_SUB;
        int64_t j0 = (ymin - VOX_SUB / 2 + VOX_SUB - 1) / VOX_SUB, j1 = (ymax - VOX_SUB / 2) / VOX_SUB;
        if (xmax < VOX_SUB / 2) i1 = -1;
        if (ymax < VOX_SUB / 2) j1 = -1;
        if (i0 < 0) i0 = 0;
        if (j0 < 0) j0 = 0;
        if (i1 > W - 1) i1 = W - 1;
        if (j1 > H - 1) j1 = H - 1;
        const int oab = owns(B->X - A->X, B->Y - A->Y), obc = owns(C->X - B->X, C->Y - B->Y),
                  oca = owns(A->X - C->X, A->Y - C->Y);
        /* mode 0: the provoking vertex is the triangle's last one (voxel.geom emits 0,1,2) */
        int64_t lo0 = 0, n0 = 0;
        if (mode == 0) {
            float lay = q[2].layer, zc = q[2].z;
            if (!(lay >= 0.0f) || lay >= (float)f.layers) continue;
            n0 = zc > 0.0f ? (int64_t)zc : 0;
            if (n0 > 128) n0 = 128;
            lo0 = 128 * (int64_t)lay;
        }
        for (int64_t j = j0; j <= j1; ++j)
            for (int64_t i = i0; i <= i1; ++i) {
                const int64_t px = i * VOX_SUB + VOX_SUB / 2, py = j * VOX_SUB + VOX_SUB / 2;
                const int64_t e0 = edge_fn(B->X, B->Y, C->X, C->Y, px, py);  /* weight of A */
                const int64_t e1 = edge_fn(C->X, C->Y, A->X, A->Y, px, py);  /* weight of B */
                const int64_t e2 = edge_fn(A->X, A->Y, B->X, B->Y, px, py);  /* weight of C */
                if (!(e0 > 0 || (e0 == 0 && obc))) continue;
                if (!(e1 > 0 || (e1 == 0 && oca))) continue;
                if (!(e2 > 0 || (e2 == 0 && oab))) continue;
                int64_t lo = lo0, n = n0;
                if (mode == 1) {
                    double zc = ((double)e0 * (double)A->z + (double)e1 * (double)B->z + (double)e2 * (double)C->z) /
                                (double)area;
                    double t = ceil(zc - 0.5);
                    n = t <= 0.0 ? 0 : (t >= (double)D ? D : (int64_t)t);
                    lo = 0;
                }
                if (n > 0) xor_range(cols + ((size_t)j * W + i) * f.words, lo, lo + n);
            }
    }
    for (int z = 0; z < D; ++z)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const uint32_t *col = cols + ((size_t)y * W + x) * f.words;
                inside[((size_t)z * H + y) * W + x] = (uint8_t)((col[z >> 5] >> (z & 31)) & 1u);
            }
    free(cols);
    return 0;
}
