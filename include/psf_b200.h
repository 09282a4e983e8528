/*
 * psf_b200.h -- C ABI of the B200 spectral-fluid step engine.
 *
 * This is the drop-in boundary for the per-step hot path of
 * ParallelSpectralFluids3D.  The reference binds that path through the C++
 * virtual interface AbstractSolver (Solver/abstractsolver.h:13-127) with two
 * implementations, PSFSolver (CPU, Solver/SolverImpl/psfsolver.cpp) and
 * PSFSolverGPU (OpenCL, Solver/SolverImpl/psfsolvergpu.cpp).  The C++ class
 * PSFSolverCUDA (include/psf/psfsolvercuda.h) implements the same interface on
 * top of these entry points; other hosts (Python ctypes, any FFI) bind them
 * directly.
 *
 * Conventions
 *   - Every entry point returns an int status: 0 on success, a negative
 *     PSF_ERR_* code otherwise.  None of them throws or exits; the message of
 *     the last failure on the calling thread is returned by psf_last_error().
 *   - A context owns all device memory it allocates; the caller owns every
 *     host buffer it passes in or out.  Host buffers may be pageable or
 *     pinned (pinned transfers overlap better).
 *   - A context is bound to one device and one CUDA stream and is not
 *     thread-safe; distinct contexts may be used from distinct threads.
 *   - Arrays are little-endian, row-major, with the sizes stated per field.
 */
#ifndef PSF_B200_H
#define PSF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSF_ABI_VERSION 1

/* Status codes. */
#define PSF_OK 0
#define PSF_ERR_INVALID -1     /* bad argument, size mismatch, null pointer */
#define PSF_ERR_CUDA -2        /* a CUDA runtime call failed */
#define PSF_ERR_NOMEM -3       /* device allocation failed */
#define PSF_ERR_SIGNS -4       /* the sign string does not fold into per-face signs */
#define PSF_ERR_STATE -5       /* call out of order (e.g. stepping before psf_set_state) */
#define PSF_ERR_UNSUPPORTED -6 /* size or option outside what the build supports */
#define PSF_ERR_TIMEOUT -7     /* a bounded device wait gave up */

/* Particle integrators.  The reference advances particles with forward
 * Euler (psfsolver.cpp:214-215, simulation.cl:203); RK4 is an extension with
 * the same interpolant and the same box clamp on every stage. */
#define PSF_RK1 1
#define PSF_RK4 4

/* Step flags. */
#define PSF_FLAG_RENORM 1u    /* w *= sqrt(e_before / e_after) (psfsolver.cpp:47-49) */
#define PSF_FLAG_DECAY_NEG 2u /* decay exp(-nu lam dt) as simulation.cl:211; default
                                 exp(+nu lam dt) as psfsolver.cpp:54 */
#define PSF_FLAG_FORCING 4u   /* w += dt * f after decay (psfsolver.cpp:56-59) */

/* Storage precision of C and Phi for a context. */
#define PSF_PRECISION_FP32 0     /* C, Phi FP32; state FP64 */
#define PSF_PRECISION_BF16X2 1   /* C, Phi as BF16 hi + lo pairs; state FP64 */

/* Voxel grid and domain box (DECMesh3D dims/resolution, Model AABB). */
typedef struct psf_grid {
    uint32_t dims[3];   /* voxels along x, y, z */
    double resolution;  /* voxel size h */
    float aabb_min[3];  /* particle box, also the grid origin */
    float aabb_max[3];
} psf_grid;

/*
 * Spectral basis of one domain (AbstractSolver members velBasisField,
 * advection, eigenValues and the DECMesh3D sign string,
 * Solver/abstractsolver.h:118-123).  All pointers are host pointers and are
 * only read during the call that receives the descriptor.
 */
typedef struct psf_basis_desc {
    psf_grid grid;
    int32_t n_modes;              /* N */
    int64_t n_active;             /* rows of phi: faces with two fluid voxels */
    const int32_t *active_faces;  /* [n_active] face ids in the reference numbering */
    const double *phi;            /* [n_active][N]  Phi restricted to active faces */
    const double *advection;      /* [N][N][N]      C[k][a][j] = advection[k](a, j) */
    const double *eigenvalues;    /* [N] */
    const uint32_t *sign_bits;    /* [ceil(V/5)] DECMesh3D::signBitString */
} psf_basis_desc;

/* Per-context step parameters (AbstractSolver setters, abstractsolver.h:24-31). */
typedef struct psf_params {
    double timestep;     /* dt */
    double viscosity;    /* nu */
    float lifetime;      /* particle lifetime given to respawned particles */
    int32_t integrator;  /* PSF_RK1 or PSF_RK4 */
    uint32_t flags;      /* PSF_FLAG_* */
    int32_t precision;   /* PSF_PRECISION_* (fixed at creation) */
    uint64_t seed;       /* respawn generator seed */
} psf_params;

typedef struct psf_ctx psf_ctx;

/* Library ABI version (PSF_ABI_VERSION of the build). */
int psf_abi_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char *psf_last_error(void);

/* Number of visible CUDA devices (0 when none). */
int psf_device_count(int *count);

/*
 * Create a single-instance context on `device`: uploads the basis in the
 * layout of the chosen precision and folds the tracer's face signs
 * (psfsolver.cpp:160-188) into Phi.  Replaces PSFSolverGPU's constructor and
 * buildAdvection uploads (psfsolvergpu.cpp:24-214, 598-874).
 */
int psf_create(const psf_basis_desc *basis, const psf_params *params, int device, psf_ctx **out);
int psf_destroy(psf_ctx *ctx);

int psf_set_params(psf_ctx *ctx, const psf_params *params);

/* Coefficient state w (AbstractSolver::basisCoeff), FP64 [n].  Setters have
 * read the caller's buffer when they return; the device work they queue
 * finishes on the context's stream before any later call's work. */
int psf_set_state(psf_ctx *ctx, const double *w, int32_t n);
int psf_get_state(psf_ctx *ctx, double *w, int32_t n);

/* Forcing vector f, FP64 [n]; applied as w += dt f when PSF_FLAG_FORCING is
 * set (the reference's projected gravity, psfsolver.cpp:344-358). */
int psf_set_forcing(psf_ctx *ctx, const double *f, int32_t n);

/* Particles as float4 (x, y, z, life), [count][4] (Graphics/Particle/Particle.h:14). */
int psf_set_particles(psf_ctx *ctx, const float *xyzw, int64_t count);
int psf_get_particles(psf_ctx *ctx, float *xyzw, int64_t count);

/* Face velocities u = float(Phi w) in the reference face numbering and sign
 * convention (AbstractSolver::velocityField), [n_faces]. */
int psf_get_velocity(psf_ctx *ctx, float *u, int64_t n_faces);

/*
 * Enqueue `nsteps` steps on the context stream (asynchronous).  One step is
 * PSFSolver::integrate (psfsolver.cpp:21-234): contraction, Euler update,
 * renormalisation, decay, forcing, reconstruction, particle tracing.
 */
int psf_step(psf_ctx *ctx, int32_t nsteps);

/* Wait for all work enqueued on the context. */
int psf_sync(psf_ctx *ctx);

/* The context's cudaStream_t, for callers that time or order work with it. */
int psf_get_stream(psf_ctx *ctx, void **stream);

/* Number of kernels one psf_step(ctx, 1) launches. */
int psf_kernels_per_step(psf_ctx *ctx, int32_t *count);

/*
 * Run one step with each kernel launched on its own between CUDA events and
 * return the device time of every kernel in milliseconds, in launch order
 * (contraction + state update, reconstruction, tracing); `n` is the capacity
 * of `kernel_ms`.  Blocks until the step is done.  This is the per-phase
 * timing of the reference's benchmark mode (t_advect_ms, t_particles_ms;
 * Solver/abstractsolver.cpp:252-302, psfsolver.cpp:62-67, 225-231).
 */
int psf_profile_step(psf_ctx *ctx, double *kernel_ms, int32_t n);

/*
 * Allocation-free coefficient step.  No counterpart in the reference: it is
 * for hosts that cannot let a library call cudaMalloc -- a real-time frame
 * loop that cannot take the device-wide stall an allocation may cause, or an
 * embedding application that owns all device memory in its own pool and only
 * passes device pointers.
 *
 * Runs one contraction + FP64 state update (the coefficient half of
 * psf_step: psfsolver.cpp:34-59) on the caller's device buffers, enqueued on
 * `stream` (a cudaStream_t, 0 for the legacy default stream) of the current
 * device:
 *   advection_f32  device, FP32 [N][N][Np] with Np = round_up(N, 4),
 *                  C[k][a][j] at (k * N + a) * Np + j, padding ignored
 *   w              device, FP64 [N], read and overwritten with the new state
 *   eigenvalues    device, FP64 [N]
 *   forcing        device, FP64 [N]; may be NULL unless PSF_FLAG_FORCING
 *   params         host; timestep, viscosity and flags are used
 * The kernel's scratch lives in a fixed array of PSF_STATIC_SCRATCH_BYTES in
 * the library's device data, held by every GPU that loads the library until
 * the process exits.  N is limited to PSF_STATIC_MAX_MODES (larger sizes
 * return PSF_ERR_UNSUPPORTED).  The first call in each CUDA context (on
 * each device, and again after cudaDeviceReset or with another context made
 * current) looks up that array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture: made while `stream` is
 * capturing, it returns PSF_ERR_STATE and enqueues nothing.  The function never calls
 * cudaMalloc or cudaFree.  All calls share the one array: calls whose
 * kernels may overlap on the GPU (unordered streams or threads) race and
 * corrupt each other's results, so order them on one stream.
 */
#define PSF_STATIC_MAX_MODES 1024
#define PSF_STATIC_SCRATCH_BYTES (4096 * 8 + 128)
int psf_coeff_step_static(const float *advection_f32, int32_t n_modes, double *w, const double *eigenvalues,
                          const double *forcing, const psf_params *params, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PSF_B200_H */
