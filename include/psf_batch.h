/*
 * psf_batch.h -- C ABI of the batched (many-instance) spectral-fluid engine.
 *
 * The reference steps one instance per solver object
 * (AbstractSolver::integrate, Solver/abstractsolver.h:18; one OpenCL queue,
 * Solver/SolverImpl/psfsolvergpu.cpp:216-256).  A batch steps many instances
 * ("slots") at once: every slot of a basis shares that basis' C and Phi,
 * which are read once per step by tensor-core GEMMs whose narrow operand is
 * the slots' coefficient vectors.  Slots may use fewer modes than their basis
 * (a prefix slice, zero-padded exactly), and have their own dt, viscosity,
 * flags, integrator, forcing, state and particles.
 *
 * Precision (PSF_PRECISION_BF16X2): C and Phi are stored as BF16 hi + lo
 * pairs, the state as BF16 hi + lo for the products, each product is
 * compensated (hi*hi + hi*lo + lo*hi) with FP32 accumulation; the state
 * update and the energy renormalisation are FP64.
 *
 * Conventions as in psf_b200.h: int status returns, host buffers owned by
 * the caller, one CUDA stream per batch, not thread-safe.
 */
#ifndef PSF_BATCH_H
#define PSF_BATCH_H

#include "psf_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PSF_BATCH_MAX_BASES 6
#define PSF_BATCH_MAX_SLOTS 256

/* One basis of a batch and the slots it serves. */
typedef struct psf_batch_basis {
    psf_basis_desc basis;     /* host arrays, read during psf_batch_create */
    int32_t slots;            /* instance slots on this basis, 1..PSF_BATCH_MAX_SLOTS */
    int64_t max_particles;    /* particle capacity of each slot */
} psf_batch_basis;

typedef struct psf_batch_config {
    int32_t n_bases;                 /* 1..PSF_BATCH_MAX_BASES */
    const psf_batch_basis *bases;
    int32_t precision;               /* PSF_PRECISION_BF16X2 */
    int32_t autotune;                /* 1: time the kernel variants at creation and keep the fastest */
    int32_t gemm_columns;            /* 0, or force the GEMM variant: 64, 128 or 256 */
    int32_t gemm_ctas;               /* 0 (one per SM), or force the persistent grid size */
    int64_t particle_pool;           /* particles resident at once over all slots (device pool);
                                        0 = every slot at its max_particles */
    int32_t contraction_ksplit;      /* 0 (1, or the autotuner's choice), or force 1, 2 or 4 K ranges
                                        per contraction row tile */
    int32_t unfused;                 /* 0: one cooperative tensor-core launch per step (contraction,
                                        state update, reconstruction); 1: three launches */
} psf_batch_config;

/* One instance placed in a slot. */
typedef struct psf_instance_desc {
    int32_t n_modes;          /* <= the basis' n_modes: the lowest n_modes modes */
    psf_params params;        /* timestep, viscosity, lifetime, integrator, flags, seed */
    const double *w0;         /* [n_modes] initial coefficients */
    const double *forcing;    /* [n_modes] or NULL */
    const float *particles;   /* [n_particles][4] (x, y, z, life) or NULL */
    int64_t n_particles;      /* <= the basis' max_particles */
    int32_t steps;            /* > 0: the slot stops advancing after this many steps; 0: no limit */
} psf_instance_desc;

typedef struct psf_batch psf_batch;

/* Kernel variant the batch runs (chosen by the autotuner or forced). */
typedef struct psf_batch_info {
    int32_t gemm_columns;      /* MMA N capacity per accumulator: 64, 128 or 256 */
    int32_t gemm_ctas;         /* persistent CTAs of the GEMM kernels */
    int32_t trace_ctas;        /* persistent CTAs of the tracer */
    int32_t kernels_per_step;  /* launches per psf_batch_step(b, 1) */
    int64_t device_bytes;      /* device memory held by the batch */
    double tuned_ms;           /* GEMM time of the chosen variant at tuning (0 if not tuned) */
    int32_t contraction_ksplit; /* K ranges per contraction row tile (1, 2 or 4) */
} psf_batch_info;

int psf_batch_create(const psf_batch_config *cfg, int device, psf_batch **out);
int psf_batch_destroy(psf_batch *b);
int psf_batch_info_get(psf_batch *b, psf_batch_info *info);

/* Place an instance in slot `slot` of basis `basis` (replaces what was there),
 * or empty the slot.  Ordered on the batch stream; returns when done.  The
 * instance's particles take a range of the batch's particle pool; if the
 * pool has no free range of that size the call fails with PSF_ERR_NOMEM and
 * the slot is left empty. */
int psf_batch_set_instance(psf_batch *b, int32_t basis, int32_t slot, const psf_instance_desc *inst);
int psf_batch_clear_instance(psf_batch *b, int32_t basis, int32_t slot);

/* The same for n placements or removals with one synchronisation; status[i]
 * receives each placement's own result (PSF_ERR_NOMEM when its particles do
 * not fit the pool, and so on). */
int psf_batch_set_instances(psf_batch *b, int32_t n, const int32_t *basis, const int32_t *slot,
                            const psf_instance_desc *const *inst, int32_t *status);
int psf_batch_clear_instances(psf_batch *b, int32_t n, const int32_t *basis, const int32_t *slot);

/* Copy the state (w[i], n_modes doubles) and the particles (xyzw[i], in the
 * caller's original order) of n occupied slots; either pointer may be NULL. */
int psf_batch_read_instances(psf_batch *b, int32_t n, const int32_t *basis, const int32_t *slot, double *const *w,
                             float *const *xyzw);

/* Free particles in the pool, and the largest contiguous free range. */
int psf_batch_pool_free(psf_batch *b, int64_t *free_particles, int64_t *largest_range);

/* Enqueue `nsteps` steps of every occupied slot (asynchronous, graph replay);
 * slots that reached their step limit do not advance. */
int psf_batch_step(psf_batch *b, int32_t nsteps);
int psf_batch_sync(psf_batch *b);
int psf_batch_get_stream(psf_batch *b, void **stream);

/* Per-slot results (synchronising). */
int psf_batch_get_state(psf_batch *b, int32_t basis, int32_t slot, double *w, int32_t n);
int psf_batch_get_particles(psf_batch *b, int32_t basis, int32_t slot, float *xyzw, int64_t count);
/* The face velocities of the slot's state as of its last step (the field its
 * particles were last traced with; none before a slot's first step). */
int psf_batch_get_velocity(psf_batch *b, int32_t basis, int32_t slot, float *u, int64_t n_faces);
int psf_batch_get_steps(psf_batch *b, int32_t basis, int32_t slot, int64_t *steps);

/* One step, run as psf_batch_step runs it, with each launch timed between
 * CUDA events (milliseconds): [tensor-core step, tracer] for a fused batch,
 * [contraction, state update, reconstruction, tracer] otherwise. */
int psf_batch_profile_step(psf_batch *b, double *kernel_ms, int32_t n);
/* One step as three tensor-core launches plus the tracer, each timed
 * (milliseconds): [contraction, state update, reconstruction, tracer]. */
int psf_batch_profile_phases(psf_batch *b, double *kernel_ms, int32_t n);

/* Device error word of the tensor-core kernels: 0, or the code of a bounded
 * wait that gave up (the batch must then be destroyed). */
int psf_batch_device_status(psf_batch *b, int32_t *code);

#ifdef __cplusplus
}
#endif

#endif /* PSF_BATCH_H */
