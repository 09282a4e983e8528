/*
 * psf_volume.h -- C ABI of the particle density volume and its ray-marched
 * image, headless (device buffers; images are returned to the caller).
 *
 * Replaces the compute part of PSFSolverGPU::drawParticles
 * (Solver/SolverImpl/psfsolvergpu.cpp:876-1022), which the reference runs
 * through OpenGL after every step:
 *   - a histogram of particle positions over the model's AABB into an R32I
 *     R^3 texture (R = 256, Solver/abstractsolver.cpp:131-141), cleared each
 *     frame (psfsolvergpu.cpp:893-900);
 *   - density = count / 1e6 stored as FP16 (Resources/Volume/volume.comp);
 *   - a per-pixel ray march with shadow rays toward a point light
 *     (Resources/Effects/Volume/volume.frag, volume.vert), output
 *     (light_energy.rgb, transmittance) per pixel.
 * The window, framebuffers and the 8-frame history blend (blit.frag) are the
 * GUI's and are not part of this library.
 *
 * The reference's histogram shader (Res/Volume/history.comp) is not in its
 * source tree; cells here are floor((p - aabb_min) / aabb_extent * R), and
 * particles outside the box are dropped.  The sampler is trilinear with
 * clamp-to-border 0 in FP32, exp(-y) on [0, 1] is a degree-12 Taylor
 * polynomial, and all arithmetic is round-to-nearest FP32 in a fixed order.
 *
 * Every entry point returns PSF_OK or a negative PSF_ERR_* code (psf_b200.h).
 */
#ifndef PSF_VOLUME_H
#define PSF_VOLUME_H

#include "psf_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PSF_VOLUME_MAX_RES 512

typedef struct psf_volume psf_volume;

/* Camera of one image (the uniforms of volume.frag / volume.vert). */
typedef struct psf_volume_view {
    float view[16];      /* view_mat, column-major (glm layout) */
    float camera[3];     /* camera_position, world space */
    float light[3];      /* light.pos, world space; the shader uses view_mat * light.pos */
    int32_t width;       /* viewport_size.z */
    int32_t height;      /* viewport_size.w */
} psf_volume_view;

/* A density volume of res^3 cells (the reference uses 256) on `device`. */
int psf_volume_create(int device, int32_t res, psf_volume **out);
int psf_volume_destroy(psf_volume *v);

/* Rebuild the density from particles (host array [n][4] = x, y, z, life)
 * over the box [aabb_min, aabb_max]. */
int psf_volume_splat(psf_volume *v, const float *particles, int64_t n, const float aabb_min[3],
                     const float aabb_max[3]);

/* Rebuild the density from a context's resident particles over its grid's
 * AABB, on the device, ordered after the context's queued steps. */
int psf_volume_splat_context(psf_volume *v, psf_ctx *ctx);

/* Copy the FP16 density (res^3 values, x fastest) to the host. */
int psf_volume_get_density(psf_volume *v, uint16_t *density, int64_t count);

/* Ray-march one image of the current density: rgba [height][width][4]
 * (row 0 = bottom row, as gl_FragCoord counts). */
int psf_volume_render(psf_volume *v, const psf_volume_view *view, float *rgba, int64_t count);

/* Device time (ms, mean of `iters`) of rebuilding the density from the
 * particles of the last splat and of rendering `view`. */
int psf_volume_profile(psf_volume *v, const psf_volume_view *view, int32_t iters, double *splat_ms,
                       double *render_ms);

#ifdef __cplusplus
}
#endif

#endif /* PSF_VOLUME_H */
