/*
 * Test infrastructure (oracle): CPU restatement of the reference's particle
 * density volume and its ray-marched rendering, used only by tests/ and by
 * bench.py's CPU baseline leg.
 *
 * Reference (PSFSolverGPU::drawParticles, Solver/SolverImpl/psfsolvergpu.cpp:876-1022):
 *   1. histogram: every particle adds 1 to the R32I cell of a 256^3 texture
 *      over the model's AABB (dispatch at :896-900; the compute shader
 *      Res/Volume/history.comp is not in the reference tree, so the binning
 *      rule -- cell = floor((p - aabb_min) / aabb_extent * R), particles
 *      outside the box dropped -- is this project's reading of its uniforms);
 *   2. density: volume = histogram / 1e6 stored as R16F
 *      (Resources/Volume/volume.comp:9-17, texture formats at
 *      Graphics/Texture3D/Texture3D.cpp:91,120; the texture is cleared each
 *      frame, :893);
 *   3. ray march per pixel (Resources/Effects/Volume/volume.frag:27-98, light
 *      position from volume.vert:17-21): ray through the pixel centre, slab
 *      test against the AABB, march in texture coordinates with
 *      step = extent.x / 256, shadow ray of up to 128 steps toward the light
 *      where the density exceeds 0.001, front-to-back emission/absorption,
 *      output (light_energy.rgb, transmittance).
 *
 * The volume sampler is trilinear with clamp-to-border 0
 * (Texture3D.cpp:125-135); the weights are computed here in FP32 (GL leaves
 * their precision to the implementation).  exp(-y) on [0, 1] uses a
 * degree-12 Taylor polynomial in Horner form.  The shader's constants
 * -1/tan(45.0/2.0) (radians) and -log(0.001) are the decimal literals below,
 * rounded to FP32 by the compiler.  Built with -ffp-contract=off: every rounding step is the
 * written one, and the CUDA kernels perform the same operations in the same
 * order, so the two agree bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct {
    float view[16];     /* column-major view matrix */
    float camera[3];
    float light[3];     /* light.pos, world space */
    float aabb_min[3], aabb_max[3];
    int32_t width, height, res;
} psfo_view;

void psfo_volume_histogram(const float *p, int64_t n, const float *mn, const float *mx, int32_t R, int32_t *hist)
{
    for (int64_t i = 0; i < n; ++i) {
        int c[3], ok = 1;
        for (int a = 0; a < 3; ++a) {
            const float ext = mx[a] - mn[a];
            const float t = (p[4 * i + a] - mn[a]) / ext;
            const float f = floorf(t * (float)R);
            if (!(f >= 0.0f) || f >= (float)R) ok = 0;
            else c[a] = (int)f;
        }
        if (ok) hist[((int64_t)c[2] * R + c[1]) * R + c[0]] += 1;
    }
}

void psfo_volume_density(const int32_t *hist, int64_t cells, _Float16 *vol)
{
    for (int64_t i = 0; i < cells; ++i) vol[i] = (_Float16)((float)hist[i] / 1000000.0f);
}

static float texel(const _Float16 *vol, int R, int x, int y, int z)
{
    if (x < 0 || y < 0 || z < 0 || x >= R || y >= R || z >= R) return 0.0f;
    return (float)vol[((int64_t)z * R + y) * R + x];
}

static float lerp1(float a, float b, float t) { return (1.0f - t) * a + t * b; }

static float sample(const _Float16 *vol, int R, float px, float py, float pz)
{
    const float u = px * (float)R - 0.5f, v = py * (float)R - 0.5f, w = pz * (float)R - 0.5f;
    const float fu = floorf(u), fv = floorf(v), fw = floorf(w);
    /* every texel outside the volume reads the border value 0 (also non-finite positions) */
    if (!(fu >= -1.0f && fu < (float)R && fv >= -1.0f && fv < (float)R && fw >= -1.0f && fw < (float)R))
        return 0.0f;
    const float a = u - fu, b = v - fv, c = w - fw;
    const int x = (int)fu, y = (int)fv, z = (int)fw;
    const float c00 = lerp1(texel(vol, R, x, y, z), texel(vol, R, x + 1, y, z), a);
    const float c10 = lerp1(texel(vol, R, x, y + 1, z), texel(vol, R, x + 1, y + 1, z), a);
    const float c01 = lerp1(texel(vol, R, x, y, z + 1), texel(vol, R, x + 1, y, z + 1), a);
    const float c11 = lerp1(texel(vol, R, x, y + 1, z + 1), texel(vol, R, x + 1, y + 1, z + 1), a);
    const float c0 = lerp1(c00, c10, b), c1 = lerp1(c01, c11, b);
    return lerp1(c0, c1, c);
}

/* exp(-y) for y in [0, 1]: Taylor series to degree 12, Horner form. */
float psfo_exp_neg_unit(float y)
{
    const float x = -y;
    float r = 1.0f;
    for (int k = 12; k >= 1; --k) r = 1.0f + (x / (float)k) * r;
    return r;
}

#define VOL_ZDIR (-1.792590986919304f)     /* -1 / tan(22.5) */
#define VOL_SHADOW_THRESH 6.907755278982137f /* -log(0.001) / 1.0 */

static float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

static float len3(float x, float y, float z) { return sqrtf((x * x + y * y) + z * z); }

void psfo_volume_render(const _Float16 *vol, const psfo_view *V, float *rgba)
{
    const int R = V->res;
    float ext[3];
    for (int a = 0; a < 3; ++a) ext[a] = V->aabb_max[a] - V->aabb_min[a];
    const float vox = ((ext[0] / (float)R) * (ext[1] / (float)R)) * (ext[2] / (float)R);
    const float step = ext[0] / 256.0f; /* step_size = extent.x / 256 (psfsolvergpu.cpp:978) */
    float lview[3]; /* view_mat * vec4(light.pos, 1) (volume.vert:19) */
    for (int i = 0; i < 3; ++i)
        lview[i] = ((V->view[i] * V->light[0] + V->view[4 + i] * V->light[1]) + V->view[8 + i] * V->light[2]) +
                   V->view[12 + i] * 1.0f;
    for (int py = 0; py < V->height; ++py)
        for (int px = 0; px < V->width; ++px) {
            float r[3];
            r[0] = 2.0f * ((float)px + 0.5f) / (float)V->width - 1.0f;
            r[1] = 2.0f * ((float)py + 0.5f) / (float)V->height - 1.0f;
            r[0] = r[0] * ((float)V->width / (float)V->height);
            r[2] = VOL_ZDIR;
            float d[3];
            for (int j = 0; j < 3; ++j) {
                const float *col = V->view + 4 * j;
                d[j] = ((r[0] * col[0] + r[1] * col[1]) + r[2] * col[2]) + 0.0f * col[3];
            }
            float tt[3], tb[3];
            for (int a = 0; a < 3; ++a) {
                const float inv = 1.0f / d[a];
                tt[a] = inv * (V->aabb_max[a] - V->camera[a]);
                tb[a] = inv * (V->aabb_min[a] - V->camera[a]);
            }
            float tmin[3], tmax[3];
            for (int a = 0; a < 3; ++a) {
                tmin[a] = fminf(tt[a], tb[a]);
                tmax[a] = fmaxf(tt[a], tb[a]);
            }
            const float t0 = fmaxf(0.0f, fmaxf(fmaxf(tmin[0], tmin[1]), fmaxf(tmin[0], tmin[2])));
            const float t1 = fminf(fminf(tmax[0], tmax[1]), fminf(tmax[0], tmax[2]));
            float pos[3], ray[3];
            for (int a = 0; a < 3; ++a) {
                const float s0 = ((V->camera[a] + d[a] * t0) - V->aabb_min[a]) / ext[a];
                const float s1 = ((V->camera[a] + d[a] * t1) - V->aabb_min[a]) / ext[a];
                pos[a] = s0;
                ray[a] = s1 - s0;
            }
            float rl = len3(ray[0], ray[1], ray[2]);
            float sv[3];
            for (int a = 0; a < 3; ++a) sv[a] = (step * ray[a]) / rl;
            float trans = 1.0f, le[3] = {0.0f, 0.0f, 0.0f};
            int steps = 1024;
            while (rl > 0.0f && steps > 0) {
                const float s = sample(vol, R, pos[0], pos[1], pos[2]) / vox;
                if (s > 0.001f) {
                    float lv[3];
                    const float lx = lview[0] - pos[0], ly = lview[1] - pos[1], lz = lview[2] - pos[2];
                    const float ll = len3(lx, ly, lz);
                    lv[0] = (step * lx) / ll;
                    lv[1] = (step * ly) / ll;
                    lv[2] = (step * lz) / ll;
                    float lp[3] = {pos[0], pos[1], pos[2]};
                    float sd = 0.0f;
                    for (int i = 0; i < 128; ++i) {
                        lp[0] = lp[0] + lv[0];
                        lp[1] = lp[1] + lv[1];
                        lp[2] = lp[2] + lv[2];
                        sd = sd + sample(vol, R, lp[0], lp[1], lp[2]) / vox;
                        if (sd > VOL_SHADOW_THRESH) break;
                    }
                    const float dens = clampf(s * step, 0.0f, 1.0f);
                    const float e = psfo_exp_neg_unit(clampf(sd * step, 0.0f, 1.0f));
                    const float sh[3] = {1.0f * e, 0.5f * e, 0.0f * e};
                    for (int a = 0; a < 3; ++a) le[a] = le[a] + (sh[a] * dens) * trans;
                    trans = trans * (1.0f - dens);
                    if (trans < 0.01f) break;
                    for (int a = 0; a < 3; ++a) le[a] = clampf(le[a], 0.0f, 1.0f);
                    trans = clampf(trans, 0.0f, 1.0f);
                }
                rl = rl - step;
                for (int a = 0; a < 3; ++a) pos[a] = pos[a] + sv[a];
                --steps;
            }
            float *o = rgba + 4 * ((int64_t)py * V->width + px);
            o[0] = le[0];
            o[1] = le[1];
            o[2] = le[2];
            o[3] = trans;
        }
}
