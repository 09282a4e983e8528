/*
 * psf_voxel.h -- C ABI of the mesh voxeliser: a closed triangle mesh becomes
 * the inside flags of the simulation grid.
 *
 * Replaces `DECMesh3D Model::voxelize(float resolution)`
 * (Graphics/Model/Model.cpp:203-451, called from AbstractSolver::setMesh,
 * Solver/abstractsolver.cpp:100 and :206), which draws the mesh into an
 * OpenGL "slice map" (Resources/Voxel/voxel.vert, voxel.geom, voxel.frag)
 * with XOR blending and reads it back.  Here the same slice-map arithmetic
 * runs as CUDA kernels on the GPU with no graphics API: every triangle is
 * rasterised at pixel centres, each covered pixel toggles the bit where its
 * surface crossing lies in that pixel's voxel column, and a suffix-parity
 * scan along each column yields the inside flags.
 *
 * Modes:
 *   PSF_VOXEL_REFERENCE  the reference's output: pixel grid = width x height
 *                        over the AABB, crossing height from the triangle's
 *                        last (provoking) vertex, z counted down from the top
 *                        of the box (the reference's projection negates z),
 *                        128-slice layers chosen per triangle as voxel.geom
 *                        does;
 *   PSF_VOXEL_GEOMETRIC  pixels of the voxel size, crossing height
 *                        interpolated at the pixel centre, z counted up, a
 *                        voxel inside when its centre is inside the surface.
 *
 * Rasterisation rules (fixed here; GL leaves them to the implementation):
 * vertices snap to 1/256 pixel, coverage uses exact 64-bit edge functions at
 * pixel centres, and a centre on an edge belongs to the triangle for which
 * that edge, walked in positive orientation, goes down or right.
 *
 * Every entry point returns PSF_OK or a negative PSF_ERR_* code (psf_b200.h).
 */
#ifndef PSF_VOXEL_H
#define PSF_VOXEL_H

#include "psf_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PSF_VOXEL_REFERENCE 0
#define PSF_VOXEL_GEOMETRIC 1
#define PSF_VOXEL_MAX_DIM 1023

typedef struct psf_voxel_mesh {
    const float *vertices;     /* [n_vertices][3], host */
    int64_t n_vertices;
    const uint32_t *triangles; /* [n_triangles][3] vertex indices, host */
    int64_t n_triangles;
} psf_voxel_mesh;

typedef struct psf_voxelizer psf_voxelizer;

/* Grid a mesh voxelises to, without touching a device: dims = (width,
 * height, depth) and aabb = (min xyz, max xyz) of the reference's AABB, which
 * starts at the origin and grows over the vertices (Model.cpp:73-80).
 * PSF_ERR_INVALID for a non-positive resolution or non-finite vertices,
 * PSF_ERR_UNSUPPORTED when an axis would exceed PSF_VOXEL_MAX_DIM voxels or
 * have none. */
int psf_voxel_grid(const psf_voxel_mesh *mesh, float resolution, int32_t mode, int32_t dims[3], float aabb[6]);

/* A voxeliser on `device` holding device buffers for meshes and grids up to
 * the given sizes (vertices, triangles, voxels). */
int psf_voxelizer_create(int device, int64_t max_vertices, int64_t max_triangles, int64_t max_voxels,
                         psf_voxelizer **out);
int psf_voxelizer_destroy(psf_voxelizer *v);

/* Upload the mesh, voxelise it and copy the inside flags (1 inside, 0
 * outside) into `inside` [depth][height][width] (voxel id z*W*H + y*W + x,
 * DEC/decmesh3d.cpp:12-15).  dims and aabb as psf_voxel_grid.  A triangle
 * index >= n_vertices is PSF_ERR_INVALID; zero-area triangles draw nothing.
 * `capacity` is the size of `inside` in bytes. */
int psf_voxelizer_run(psf_voxelizer *v, const psf_voxel_mesh *mesh, float resolution, int32_t mode,
                      int32_t dims[3], float aabb[6], uint8_t *inside, int64_t capacity);

/* Re-run the device part of the last psf_voxelizer_run `iters` times on the
 * resident mesh and report the mean device time of one voxelisation (ms). */
int psf_voxelizer_profile(psf_voxelizer *v, int32_t iters, double *ms);

/* One-shot form: create, run, destroy. */
int psf_voxelize(const psf_voxel_mesh *mesh, float resolution, int32_t mode, int device, int32_t dims[3],
                 float aabb[6], uint8_t *inside, int64_t capacity);

#ifdef __cplusplus
}
#endif

#endif /* PSF_VOXEL_H */
