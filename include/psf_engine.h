/*
 * psf_engine.h -- C ABI of the serving engine: continuous batching of
 * spectral-fluid rollouts on one GPU.
 *
 * The reference runs one rollout at a time from its GUI timer
 * (Widgets/glcanvas.cpp:143-156 -> AbstractSolver::integrate).  The engine
 * instead accepts rollout requests from any thread at any time.  A worker
 * thread admits queued requests into free slots of a batch (psf_batch.h)
 * whenever a slot, a particle range and the device-memory budget allow,
 * steps every admitted rollout together, and retires each one when its own
 * step count is reached, so requests that arrive while others run join the
 * next step.  Each rollout's state, face field and particles stay on the
 * device from admission to completion; the per-domain C and Phi are shared.
 *
 * Every entry point returns 0 or a negative PSF_ERR_* code (psf_b200.h).
 * psf_engine_submit, _poll, _wait, _collect and _stats_get may be called
 * from any thread.
 */
#ifndef PSF_ENGINE_H
#define PSF_ENGINE_H

#include "psf_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct psf_engine psf_engine;

typedef struct psf_engine_config {
    int32_t n_bases;                 /* domains, 1..PSF_BATCH_MAX_BASES */
    const psf_basis_desc *bases;     /* host arrays, read during create */
    const int32_t *slots;            /* [n_bases] concurrent rollouts per domain */
    int64_t max_particles;           /* largest particle count of one rollout */
    int64_t particle_pool;           /* particles resident at once (0: every slot at max_particles) */
    int64_t hbm_budget_bytes;        /* device bytes the admitted rollouts may hold (0: no limit) */
    int32_t chunk_steps;             /* steps launched between admission rounds (0: 8) */
    int32_t autotune;                /* 1: tune the GEMM variant at create */
} psf_engine_config;

/* One rollout: `steps` steps of the reference update from w0 on the lowest
 * n_modes modes of basis `basis`, with its particles. */
typedef struct psf_request {
    int32_t basis;
    int32_t n_modes;
    int32_t steps;
    int32_t reserved;
    psf_params params;
    const double *w0;         /* [n_modes], copied at submit */
    const double *forcing;    /* [n_modes] or NULL, copied at submit */
    const float *particles;   /* [n_particles][4] or NULL, copied at submit */
    int64_t n_particles;
} psf_request;

/* Timeline of a finished request, in seconds since the engine was created. */
typedef struct psf_request_info {
    uint64_t id;
    int32_t status;           /* PSF_OK, or the error that ended the request */
    int32_t steps;
    double t_submit;
    double t_admit;
    double t_done;
} psf_request_info;

typedef struct psf_engine_stats {
    int64_t submitted, admitted, completed, queued, active;
    int64_t instance_steps;   /* rollout steps completed */
    int64_t particle_steps;
    int64_t step_launches;    /* batch steps launched */
    int64_t budget_refusals;  /* admission attempts deferred for lack of budget, slots or pool */
    int64_t device_bytes;     /* held by the engine's batch */
    int64_t rollout_bytes;    /* of which charged to admitted rollouts */
    double t_now;
    double step_s;            /* worker wall time in step launches and their synchronisation */
    double admit_s;           /* worker wall time placing admitted rollouts */
    double retire_s;          /* worker wall time copying out and clearing finished rollouts */
} psf_engine_stats;

int psf_engine_create(const psf_engine_config *cfg, int device, psf_engine **out);
/* Stops the worker after its current chunk; unfinished requests are dropped. */
int psf_engine_destroy(psf_engine *e);

/* Queue a rollout (inputs are copied); returns its id.  PSF_ERR_INVALID for
 * a request that can never be admitted (unknown basis, too many modes or
 * particles, larger than the whole budget). */
int psf_engine_submit(psf_engine *e, const psf_request *req, uint64_t *id);

/* Ids of finished requests not yet collected (up to `max`). */
int psf_engine_poll(psf_engine *e, uint64_t *ids, int32_t max, int32_t *n);
/* Block until request `id` finished (PSF_OK) or `timeout_s` passed (PSF_ERR_TIMEOUT). */
int psf_engine_wait(psf_engine *e, uint64_t id, double timeout_s);
/* Copy a finished request's final state and particles (either may be NULL)
 * and its timeline, then forget it. */
int psf_engine_collect(psf_engine *e, uint64_t id, double *w, int32_t n, float *particles, int64_t count,
                       psf_request_info *info);
/* Block until nothing is queued or running, or `timeout_s` passed. */
int psf_engine_drain(psf_engine *e, double timeout_s);
int psf_engine_stats_get(psf_engine *e, psf_engine_stats *stats);

#ifdef __cplusplus
}
#endif

#endif /* PSF_ENGINE_H */
