// Serving engine (include/psf_engine.h): continuous batching of rollouts.
//
// One worker thread owns a psf_batch.  Each round it admits queued requests
// (first come first served, skipping requests that do not fit yet) into free
// slots while the slot count, the particle pool and the device-memory budget
// allow, launches a chunk of steps for every admitted rollout (a rollout
// stops on the device at its own step count), and retires finished rollouts
// by copying their state and particles out and freeing their slot.  Callers
// submit, poll, wait and collect from any thread.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "psf_b200.h"
#include "psf_batch.h"
#include "psf_engine.h"
#include "psf_internal.h"

using psf::fail;

namespace {

struct Request {
    uint64_t id = 0;
    int32_t basis = 0, n_modes = 0, steps = 0;
    psf_params params{};
    std::vector<double> w0, force;
    std::vector<float> parts;
    std::vector<double> w_out;
    std::vector<float> p_out;
    int status = PSF_OK;
    int slot = -1;
    int64_t remaining = 0;
    int64_t bytes = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
};
using ReqPtr = std::shared_ptr<Request>;

struct BasisInfo {
    int32_t n_modes = 0;
    int64_t voxels = 0;
    int32_t slots = 0;
};

}  // namespace

struct psf_engine {
    psf_batch *batch = nullptr;
    int device = 0;
    int chunk = 8;
    int64_t max_particles = 0;
    int64_t pool_cap = 0;
    int64_t budget = 0;
    std::vector<BasisInfo> bases;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<ReqPtr> queue;
    std::vector<std::vector<int>> free_slots;
    std::vector<std::vector<ReqPtr>> active;
    std::unordered_map<uint64_t, ReqPtr> done;
    std::deque<uint64_t> done_order;
    uint64_t next_id = 1;
    psf_engine_stats st{};
    int64_t rollout_bytes = 0;
    int fatal = PSF_OK;
    std::string fatal_msg;
    std::atomic<bool> stop{false};
    std::thread worker;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    // Device bytes a rollout is charged while admitted: its particles (pool
    // entry and order index), its face pairs, state and forcing.
    int64_t charge(const Request &r) const
    {
        const BasisInfo &b = bases[(size_t)r.basis];
        return (int64_t)r.parts.size() / 4 * 20 + 24 * b.voxels + 16 * (int64_t)b.n_modes;
    }
    void run();
    void finish(const ReqPtr &r, int status);
    int admit_round();
    int step_round();
};

void psf_engine::finish(const ReqPtr &r, int status)
{
    std::lock_guard<std::mutex> lock(mu);
    r->status = status;
    r->t_done = now();
    if (r->slot >= 0) {
        free_slots[(size_t)r->basis].push_back(r->slot);
        active[(size_t)r->basis][(size_t)r->slot].reset();
        rollout_bytes -= r->bytes;
        st.active -= 1;
        r->slot = -1;
    }
    done[r->id] = r;
    done_order.push_back(r->id);
    st.completed += 1;
    cv_done.notify_all();
}

int psf_engine::admit_round()
{
    std::vector<ReqPtr> picked;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (auto it = queue.begin(); it != queue.end();) {
            const ReqPtr &r = *it;
            std::vector<int> &fs = free_slots[(size_t)r->basis];
            if (fs.empty() || (budget > 0 && rollout_bytes + r->bytes > budget)) {
                st.budget_refusals += 1;
                ++it;
                continue;
            }
            r->slot = fs.back();
            fs.pop_back();
            rollout_bytes += r->bytes;
            active[(size_t)r->basis][(size_t)r->slot] = r;
            st.active += 1;
            st.queued -= 1;
            picked.push_back(r);
            it = queue.erase(it);
        }
    }
    if (picked.empty()) return PSF_OK;
    std::vector<psf_instance_desc> descs(picked.size());
    std::vector<const psf_instance_desc *> dptr(picked.size());
    std::vector<int32_t> bas(picked.size()), slt(picked.size()), status(picked.size(), PSF_OK);
    for (size_t i = 0; i < picked.size(); ++i) {
        const ReqPtr &r = picked[i];
        psf_instance_desc &d = descs[i];
        d = psf_instance_desc{};
        d.n_modes = r->n_modes;
        d.params = r->params;
        d.w0 = r->w0.data();
        d.forcing = r->force.empty() ? nullptr : r->force.data();
        d.particles = r->parts.empty() ? nullptr : r->parts.data();
        d.n_particles = (int64_t)r->parts.size() / 4;
        d.steps = r->steps;
        dptr[i] = &d;
        bas[i] = r->basis;
        slt[i] = r->slot;
    }
    const double ta = now();
    const int rc_all = psf_batch_set_instances(batch, (int32_t)picked.size(), bas.data(), slt.data(), dptr.data(),
                                               status.data());
    {
        std::lock_guard<std::mutex> lock(mu);
        st.admit_s += now() - ta;
    }
    for (size_t i = 0; i < picked.size(); ++i) {
        const ReqPtr &r = picked[i];
        const int rc = rc_all != PSF_OK ? rc_all : status[i];
        if (rc == PSF_ERR_NOMEM) {
            // No contiguous particle range yet: back to the head of the queue.
            std::lock_guard<std::mutex> lock(mu);
            free_slots[(size_t)r->basis].push_back(r->slot);
            active[(size_t)r->basis][(size_t)r->slot].reset();
            rollout_bytes -= r->bytes;
            r->slot = -1;
            st.active -= 1;
            st.queued += 1;
            st.budget_refusals += 1;
            queue.push_front(r);
            continue;
        }
        if (rc != PSF_OK) {
            finish(r, rc);
            continue;
        }
        std::lock_guard<std::mutex> lock(mu);
        r->t_admit = now();
        r->remaining = r->steps;
        st.admitted += 1;
    }
    return PSF_OK;
}

int psf_engine::step_round()
{
    std::vector<ReqPtr> running;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (auto &per : active)
            for (auto &r : per)
                if (r && r->remaining > 0) running.push_back(r);
    }
    if (running.empty()) return PSF_OK;
    int64_t most = 0;
    for (const ReqPtr &r : running) most = std::max(most, r->remaining);
    const int k = (int)std::min<int64_t>(chunk, most);
    const double ts = now();
    int rc = psf_batch_step(batch, k);
    if (rc == PSF_OK) rc = psf_batch_sync(batch);
    if (rc != PSF_OK) return rc;
    const double t_stepped = now();
    std::vector<ReqPtr> finished;
    {
        std::lock_guard<std::mutex> lock(mu);
        st.step_launches += k;
        st.step_s += t_stepped - ts;
        for (const ReqPtr &r : running) {
            const int64_t d = std::min<int64_t>(k, r->remaining);
            r->remaining -= d;
            st.instance_steps += d;
            st.particle_steps += d * ((int64_t)r->parts.size() / 4);
            if (r->remaining == 0) finished.push_back(r);
        }
    }
    if (finished.empty()) return PSF_OK;
    std::vector<int32_t> bas(finished.size()), slt(finished.size());
    std::vector<double *> wp(finished.size());
    std::vector<float *> pp(finished.size());
    for (size_t i = 0; i < finished.size(); ++i) {
        const ReqPtr &r = finished[i];
        r->w_out.resize((size_t)r->n_modes);
        r->p_out.resize(r->parts.size());
        bas[i] = r->basis;
        slt[i] = r->slot;
        wp[i] = r->w_out.data();
        pp[i] = r->p_out.empty() ? nullptr : r->p_out.data();
    }
    const double tr = now();
    int e = psf_batch_read_instances(batch, (int32_t)finished.size(), bas.data(), slt.data(), wp.data(), pp.data());
    if (e == PSF_OK) e = psf_batch_clear_instances(batch, (int32_t)finished.size(), bas.data(), slt.data());
    {
        std::lock_guard<std::mutex> lock(mu);
        st.retire_s += now() - tr;
    }
    for (const ReqPtr &r : finished) {
        r->parts.clear();
        r->parts.shrink_to_fit();
        finish(r, e);
    }
    if (e != PSF_OK) return e;
    return PSF_OK;
}

void psf_engine::run()
{
    while (!stop.load()) {
        int rc = admit_round();
        bool idle = false;
        {
            std::lock_guard<std::mutex> lock(mu);
            idle = st.active == 0;
        }
        if (idle) {
            std::unique_lock<std::mutex> lock(mu);
            cv_work.wait_for(lock, std::chrono::milliseconds(20), [&] { return stop.load() || !queue.empty(); });
            continue;
        }
        if (rc == PSF_OK) rc = step_round();
        if (rc != PSF_OK) {
            // A device error ends every admitted and queued request.
            std::vector<ReqPtr> all;
            {
                std::lock_guard<std::mutex> lock(mu);
                fatal = rc;
                fatal_msg = psf_last_error();
                for (auto &per : active)
                    for (auto &r : per)
                        if (r) all.push_back(r);
                for (auto &r : queue) all.push_back(r);
                queue.clear();
                st.queued = 0;
            }
            for (auto &r : all) finish(r, rc);
            return;
        }
    }
}

extern "C" {

int psf_engine_create(const psf_engine_config *cfg, int device, psf_engine **out)
{
    if (!cfg || !out || !cfg->bases || !cfg->slots) return fail(PSF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->n_bases < 1 || cfg->n_bases > PSF_BATCH_MAX_BASES)
        return fail(PSF_ERR_UNSUPPORTED, "n_bases must be in [1, PSF_BATCH_MAX_BASES]");
    if (cfg->max_particles < 0 || cfg->hbm_budget_bytes < 0 || cfg->chunk_steps < 0)
        return fail(PSF_ERR_INVALID, "negative size in the engine configuration");
    psf_engine *e = nullptr;
    try {
        e = new psf_engine();
    } catch (const std::bad_alloc &) {
        return fail(PSF_ERR_NOMEM, "host allocation failed");
    }
    e->device = device;
    e->chunk = cfg->chunk_steps > 0 ? cfg->chunk_steps : 8;
    e->max_particles = cfg->max_particles;
    e->budget = cfg->hbm_budget_bytes;
    std::vector<psf_batch_basis> bb((size_t)cfg->n_bases);
    for (int i = 0; i < cfg->n_bases; ++i) {
        bb[(size_t)i].basis = cfg->bases[i];
        bb[(size_t)i].slots = cfg->slots[i];
        bb[(size_t)i].max_particles = cfg->max_particles;
        BasisInfo info;
        info.n_modes = cfg->bases[i].n_modes;
        info.voxels = (int64_t)cfg->bases[i].grid.dims[0] * cfg->bases[i].grid.dims[1] * cfg->bases[i].grid.dims[2];
        info.slots = cfg->slots[i];
        e->bases.push_back(info);
    }
    psf_batch_config bc{};
    bc.n_bases = cfg->n_bases;
    bc.bases = bb.data();
    bc.precision = PSF_PRECISION_BF16X2;
    bc.autotune = cfg->autotune;
    bc.particle_pool = cfg->particle_pool;
    int rc = psf_batch_create(&bc, device, &e->batch);
    if (rc != PSF_OK) {
        delete e;
        return rc;
    }
    e->free_slots.resize((size_t)cfg->n_bases);
    e->active.resize((size_t)cfg->n_bases);
    for (int i = 0; i < cfg->n_bases; ++i) {
        for (int s = cfg->slots[i] - 1; s >= 0; --s) e->free_slots[(size_t)i].push_back(s);
        e->active[(size_t)i].resize((size_t)cfg->slots[i]);
    }
    psf_batch_info bi{};
    psf_batch_info_get(e->batch, &bi);
    e->st.device_bytes = bi.device_bytes;
    int64_t largest = 0;
    psf_batch_pool_free(e->batch, &e->pool_cap, &largest);
    try {
        e->worker = std::thread([e] {
            cudaSetDevice(e->device);
            e->run();
        });
    } catch (...) {
        psf_batch_destroy(e->batch);
        delete e;
        return fail(PSF_ERR_INVALID, "could not start the engine's worker thread");
    }
    *out = e;
    return PSF_OK;
}

int psf_engine_destroy(psf_engine *e)
{
    if (!e) return PSF_OK;
    e->stop.store(true);
    e->cv_work.notify_all();
    if (e->worker.joinable()) e->worker.join();
    psf_batch_destroy(e->batch);
    delete e;
    return PSF_OK;
}

int psf_engine_submit(psf_engine *e, const psf_request *q, uint64_t *id)
{
    if (!e || !q || !id || !q->w0) return fail(PSF_ERR_INVALID, "null argument");
    if (q->basis < 0 || q->basis >= (int32_t)e->bases.size()) return fail(PSF_ERR_INVALID, "unknown basis");
    const BasisInfo &b = e->bases[(size_t)q->basis];
    if (q->n_modes < 1 || q->n_modes > b.n_modes) return fail(PSF_ERR_INVALID, "n_modes out of range for the basis");
    if (q->steps < 1) return fail(PSF_ERR_INVALID, "steps must be >= 1");
    if (q->n_particles < 0 || q->n_particles > e->max_particles)
        return fail(PSF_ERR_INVALID, "n_particles exceeds the engine's max_particles");
    if (q->n_particles > 0 && !q->particles) return fail(PSF_ERR_INVALID, "particles is null");
    if (q->n_particles > e->pool_cap) return fail(PSF_ERR_INVALID, "n_particles exceeds the particle pool");
    if ((q->params.flags & PSF_FLAG_FORCING) && !q->forcing)
        return fail(PSF_ERR_INVALID, "PSF_FLAG_FORCING is set but forcing is null");
    if (!(q->params.timestep > 0.0)) return fail(PSF_ERR_INVALID, "timestep must be positive");
    if (q->params.integrator != PSF_RK1 && q->params.integrator != PSF_RK4)
        return fail(PSF_ERR_INVALID, "integrator must be PSF_RK1 or PSF_RK4");
    ReqPtr r;
    try {
        r = std::make_shared<Request>();
        r->basis = q->basis;
        r->n_modes = q->n_modes;
        r->steps = q->steps;
        r->params = q->params;
        r->w0.assign(q->w0, q->w0 + q->n_modes);
        if (q->forcing) r->force.assign(q->forcing, q->forcing + q->n_modes);
        if (q->n_particles > 0) r->parts.assign(q->particles, q->particles + 4 * q->n_particles);
    } catch (const std::bad_alloc &) {
        return fail(PSF_ERR_NOMEM, "host allocation failed");
    }
    r->bytes = e->charge(*r);
    if (e->budget > 0 && r->bytes > e->budget) return fail(PSF_ERR_INVALID, "request is larger than the whole budget");
    {
        std::lock_guard<std::mutex> lock(e->mu);
        if (e->fatal != PSF_OK) return fail(e->fatal, "engine stopped: " + e->fatal_msg);
        r->id = e->next_id++;
        r->t_submit = e->now();
        e->queue.push_back(r);
        e->st.submitted += 1;
        e->st.queued += 1;
        *id = r->id;
    }
    e->cv_work.notify_all();
    return PSF_OK;
}

int psf_engine_poll(psf_engine *e, uint64_t *ids, int32_t max, int32_t *n)
{
    if (!e || !n || (max > 0 && !ids)) return fail(PSF_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lock(e->mu);
    int32_t k = 0;
    for (auto it = e->done_order.begin(); it != e->done_order.end() && k < max; ++it)
        if (e->done.count(*it)) ids[k++] = *it;
    *n = k;
    return PSF_OK;
}

int psf_engine_wait(psf_engine *e, uint64_t id, double timeout_s)
{
    if (!e) return fail(PSF_ERR_INVALID, "null engine");
    std::unique_lock<std::mutex> lock(e->mu);
    const bool ok = e->cv_done.wait_for(lock, std::chrono::duration<double>(std::max(0.0, timeout_s)),
                                        [&] { return e->done.count(id) > 0; });
    return ok ? PSF_OK : fail(PSF_ERR_TIMEOUT, "request not finished before the timeout");
}

int psf_engine_collect(psf_engine *e, uint64_t id, double *w, int32_t n, float *particles, int64_t count,
                       psf_request_info *info)
{
    if (!e) return fail(PSF_ERR_INVALID, "null engine");
    ReqPtr r;
    {
        std::lock_guard<std::mutex> lock(e->mu);
        auto it = e->done.find(id);
        if (it == e->done.end()) return fail(PSF_ERR_STATE, "request not finished or already collected");
        r = it->second;
        if (w && n != r->n_modes) return fail(PSF_ERR_INVALID, "n must equal the request's n_modes");
        if (particles && count != (int64_t)r->p_out.size() / 4)
            return fail(PSF_ERR_INVALID, "count must equal the request's particle count");
        e->done.erase(it);
        auto pos = std::find(e->done_order.begin(), e->done_order.end(), id);
        if (pos != e->done_order.end()) e->done_order.erase(pos);
    }
    if (info) {
        info->id = r->id;
        info->status = r->status;
        info->steps = r->steps;
        info->t_submit = r->t_submit;
        info->t_admit = r->t_admit;
        info->t_done = r->t_done;
    }
    if (r->status == PSF_OK) {
        if (w) std::memcpy(w, r->w_out.data(), (size_t)n * 8);
        if (particles && count > 0) std::memcpy(particles, r->p_out.data(), (size_t)count * 16);
    }
    return PSF_OK;
}

int psf_engine_drain(psf_engine *e, double timeout_s)
{
    if (!e) return fail(PSF_ERR_INVALID, "null engine");
    std::unique_lock<std::mutex> lock(e->mu);
    const bool ok = e->cv_done.wait_for(lock, std::chrono::duration<double>(std::max(0.0, timeout_s)), [&] {
        return (e->queue.empty() && e->st.active == 0) || e->fatal != PSF_OK;
    });
    if (e->fatal != PSF_OK) return fail(e->fatal, "engine stopped: " + e->fatal_msg);
    return ok ? PSF_OK : fail(PSF_ERR_TIMEOUT, "requests still queued or running at the timeout");
}

int psf_engine_stats_get(psf_engine *e, psf_engine_stats *s)
{
    if (!e || !s) return fail(PSF_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lock(e->mu);
    *s = e->st;
    s->rollout_bytes = e->rollout_bytes;
    s->t_now = e->now();
    return PSF_OK;
}

}  // extern "C"
