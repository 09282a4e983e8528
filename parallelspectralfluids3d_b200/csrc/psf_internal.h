// Internal types shared by the kernels and the C ABI implementation.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "psf_b200.h"

namespace psf {

// Largest mode count a context accepts (shared-memory staging of w).
constexpr int PSF_MAX_MODES = 1024;

// Grid constants for the tracer (DECMesh3D dims and face-block offsets,
// DEC/decmesh3d.cpp:17-30).
struct GridDev {
    int nx, ny, nz;
    float inv_h;
    float mn[3];     // aabb min: grid origin and lower clamp
    float mx[3];     // aabb max: upper clamp
    float shift[3];  // aabb min + extent: the reference's index offset (psfsolver.cpp:80)
    uint32_t yoff;   // number of z-faces
    uint32_t xoff;   // number of z- and y-faces
    int centered;    // shift == -mn on every axis: the index and weight coordinates coincide
};

struct StateParams {
    double dt;
    double visc_signed;  // +nu (CPU path) or -nu (OpenCL path)
    unsigned int flags;
};

struct TraceParams {
    float dt;
    float lifetime;
    int rk4;
    unsigned long long seed;
};

// Device view of a single-instance context.
struct PlainDev {
    int N, Np, S;
    long long n_active, ldp, n_faces, P;
    const float *C;      // [N][N][Np]
    const float *phiT;   // [ldp / 64][N][64]: 64-face tiles, each mode-major; signed
    const int32_t *faces;
    // The contraction reads w (and its step count) and writes the updated
    // state to w_next (and the count + 1); the reconstruction reads w.  A
    // context keeps two state buffers and alternates them, so the next
    // step's contraction runs beside this step's reconstruction and tracer;
    // w_next == w updates in place.
    double *w, *w_next, *dwpart;
    const double *lam, *force;
    unsigned int *ticket;
    unsigned long long *step_ctr, *step_ctr_next;
    float *u;            // [n_faces], signed
    float2 *pairs;       // [3][V] per-voxel face pairs (x, y, z), signed: written by the reconstruction
    const float2 *trace_pairs;                // the face pairs the tracer reads
    const unsigned long long *trace_ctr;      // step count of the state the tracer advects with
    const int32_t *pair_dst;  // [n_active][2] float indices into pairs of each active face
    int trace_blocks;    // persistent tracer grid: SMs x resident blocks per SM
    float4 *parts;       // [P] in cell (Morton) order
    const int32_t *perm; // [P] caller index of each stored particle
    GridDev grid;
    StateParams sp;
    TraceParams tp;
};

// Scratch buffers for putting particles into cell order and back.
struct OrderBufs {
    float4 *staging = nullptr;  // [P] caller order
    uint32_t *keys_in = nullptr, *keys_out = nullptr;
    int32_t *idx_in = nullptr;
    void *temp = nullptr;
    size_t temp_bytes = 0;
};

// Number of faces of a grid in the reference numbering (z-, y-, then x-faces).
int64_t n_faces_of(const psf_grid &g);
// Sign (+1/-1) with which the reference tracer reads each face (0 for faces
// no voxel reads); PSF_ERR_SIGNS if two voxels read a face with different signs.
int fold_signs(const psf_grid &g, const uint32_t *bits, std::vector<int8_t> &sigma);

// For each active face, the two float slots of the per-voxel face-pair field
// (float view of [3][V] float2) that hold its value: one in each adjacent voxel.
void face_pair_slots(const psf_grid &g, const int32_t *faces, int64_t n_active, std::vector<int32_t> &dst);

// Tracer constants of a grid (the reference's index offsets and box).
GridDev make_grid_dev(const psf_grid &g);

// Resident particles of a single-instance context (for consumers on its device).
struct ContextParticles {
    int device;
    cudaStream_t stream;
    const float4 *parts;  // [n] in the context's storage order
    long long n;
    float mn[3], mx[3];   // the grid's AABB
};
int context_particles(psf_ctx *c, ContextParticles *out);

extern thread_local std::string g_last_error;
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

int launch_contract_state(const PlainDev &d, cudaStream_t st);
// `after_kernel`: the launch directly follows a kernel in the stream and may
// start during that kernel's tail (programmatic dependent launch).
int launch_reconstruct(const PlainDev &d, cudaStream_t st, bool after_kernel = true);
int launch_trace(const PlainDev &d, cudaStream_t st, bool after_kernel = true);
int trace_blocks_per_sm();
int sort_particles_temp_bytes(long long P, size_t *bytes);
// Put caller-order particles (o.staging) into cell order: a Morton sort that
// rewrites d.perm, or with `resort` false a gather through the current perm.
int launch_order_particles(const PlainDev &d, const OrderBufs &o, cudaStream_t st, bool resort = true);
int launch_unorder_particles(const PlainDev &d, const OrderBufs &o, cudaStream_t st);

}  // namespace psf
