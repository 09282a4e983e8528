// Serving engine (include/psf_engine.h): continuous batching of rollouts.
//
// One worker thread owns a psf_batch.  Each round launches a chunk of steps
// for every admitted rollout (a rollout stops on the device at its own step
// count) and, while that chunk runs, does the host work of the round:
//   - it retires the rollouts that reached their step count in the previous
//     chunk: their slots are no longer stepped, so their state and particles
//     are read on a second stream beside the running chunk;
//   - it picks queued requests (first come first served, skipping requests
//     that do not fit yet) for the slots, particle pool and device-memory
//     budget that are free, and copies their particles into pinned memory.
// After the chunk the retired slots are cleared and the picked requests
// placed (their uploads queued ahead of the next chunk, without waiting).
// Callers submit, poll, wait and collect from any thread.

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
#include "psf_batch_internal.h"
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
    const float *src = nullptr;  // pinned copy of `parts` for the placement, if staged
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
    // Pinned staging of picked requests' particles: two halves used by
    // alternate rounds; an event marks when the placements reading a half ran.
    float *arena = nullptr;
    int64_t arena_floats = 0;  // per half
    int half = 0;
    cudaEvent_t half_done[2] = {nullptr, nullptr};
    bool half_used[2] = {false, false};

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
    void release()
    {
        psf_batch_destroy(batch);
        batch = nullptr;
        for (cudaEvent_t &ev : half_done)
            if (ev) cudaEventDestroy(ev);
        if (arena) cudaFreeHost(arena);
        arena = nullptr;
    }
    void run();
    void finish(const ReqPtr &r, int status);
    std::vector<ReqPtr> pick();
    int stage(std::vector<ReqPtr> &picked);
    int place(std::vector<ReqPtr> &picked);
    int retire(std::vector<ReqPtr> &frozen, std::vector<int32_t> &clear_b, std::vector<int32_t> &clear_s);
    void fail_all(int rc);
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

// Queued requests that fit now, in arrival order: a free slot of their basis
// and room in the budget.  They are moved to `active` with their slot.
std::vector<ReqPtr> psf_engine::pick()
{
    std::vector<ReqPtr> picked;
    std::lock_guard<std::mutex> lock(mu);
    size_t free_total = 0;
    for (const auto &fs : free_slots) free_total += fs.size();
    for (auto it = queue.begin(); it != queue.end() && free_total > 0;) {
        const ReqPtr &r = *it;
        std::vector<int> &fs = free_slots[(size_t)r->basis];
        if (fs.empty() || (budget > 0 && rollout_bytes + r->bytes > budget)) {
            st.budget_refusals += 1;
            ++it;
            continue;
        }
        r->slot = fs.back();
        fs.pop_back();
        --free_total;
        rollout_bytes += r->bytes;
        active[(size_t)r->basis][(size_t)r->slot] = r;
        st.active += 1;
        st.queued -= 1;
        picked.push_back(r);
        it = queue.erase(it);
    }
    return picked;
}

// Copy the picked requests' particles into the pinned half of this round
// (those that do not fit are placed from their own, pageable, copy).
int psf_engine::stage(std::vector<ReqPtr> &picked)
{
    if (picked.empty() || !arena) return PSF_OK;
    if (half_used[half]) {
        cudaError_t e = cudaEventSynchronize(half_done[half]);
        if (e != cudaSuccess) return psf::cuda_fail(e, "cudaEventSynchronize");
        half_used[half] = false;
    }
    float *base = arena + (size_t)half * (size_t)arena_floats;
    int64_t used = 0;
    for (const ReqPtr &r : picked) {
        r->src = nullptr;
        const int64_t n = (int64_t)r->parts.size();
        if (n == 0 || used + n > arena_floats) continue;
        std::memcpy(base + used, r->parts.data(), (size_t)n * sizeof(float));
        r->src = base + used;
        used += n;
    }
    return PSF_OK;
}

// Place the picked requests into their slots.  The uploads, particle
// orderings and the priming contraction are queued on the batch's stream
// ahead of the next chunk; nothing waits for them here.
int psf_engine::place(std::vector<ReqPtr> &picked)
{
    if (picked.empty()) return PSF_OK;
    std::vector<psf_instance_desc> descs(picked.size());
    std::vector<const psf_instance_desc *> dptr(picked.size());
    std::vector<int32_t> bas(picked.size()), slt(picked.size()), status(picked.size(), PSF_OK);
    bool staged = false;
    for (size_t i = 0; i < picked.size(); ++i) {
        const ReqPtr &r = picked[i];
        psf_instance_desc &d = descs[i];
        d = psf_instance_desc{};
        d.n_modes = r->n_modes;
        d.params = r->params;
        d.w0 = r->w0.data();
        d.forcing = r->force.empty() ? nullptr : r->force.data();
        d.particles = r->parts.empty() ? nullptr : (r->src ? r->src : r->parts.data());
        staged |= r->src != nullptr;
        d.n_particles = (int64_t)r->parts.size() / 4;
        d.steps = r->steps;
        dptr[i] = &d;
        bas[i] = r->basis;
        slt[i] = r->slot;
    }
    const double ta = now();
    const int rc_all =
        psf::batch_place_async(batch, (int32_t)picked.size(), bas.data(), slt.data(), dptr.data(), status.data());
    if (staged) {
        void *stream = nullptr;
        psf_batch_get_stream(batch, &stream);
        cudaError_t e = cudaEventRecord(half_done[half], (cudaStream_t)stream);
        if (e != cudaSuccess) return psf::cuda_fail(e, "cudaEventRecord");
        half_used[half] = true;
        half ^= 1;
    }
    {
        std::lock_guard<std::mutex> lock(mu);
        st.admit_s += now() - ta;
    }
    for (size_t i = 0; i < picked.size(); ++i) {
        const ReqPtr &r = picked[i];
        r->src = nullptr;
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
    return rc_all == PSF_ERR_NOMEM ? PSF_OK : rc_all;
}

// Read out the rollouts that reached their step count in the previous chunk
// (their slots are not stepped by the chunk now running) and complete them;
// their slots are cleared once the running chunk is done.
int psf_engine::retire(std::vector<ReqPtr> &frozen, std::vector<int32_t> &clear_b, std::vector<int32_t> &clear_s)
{
    if (frozen.empty()) return PSF_OK;
    std::vector<int32_t> bas(frozen.size()), slt(frozen.size());
    std::vector<double *> wp(frozen.size());
    std::vector<float *> pp(frozen.size());
    for (size_t i = 0; i < frozen.size(); ++i) {
        const ReqPtr &r = frozen[i];
        r->w_out.resize((size_t)r->n_modes);
        r->p_out.resize(r->parts.size());
        bas[i] = r->basis;
        slt[i] = r->slot;
        wp[i] = r->w_out.data();
        pp[i] = r->p_out.empty() ? nullptr : r->p_out.data();
    }
    const double tr = now();
    const int e = psf::batch_read_frozen(batch, (int32_t)frozen.size(), bas.data(), slt.data(), wp.data(), pp.data());
    {
        std::lock_guard<std::mutex> lock(mu);
        st.retire_s += now() - tr;
    }
    clear_b.insert(clear_b.end(), bas.begin(), bas.end());
    clear_s.insert(clear_s.end(), slt.begin(), slt.end());
    for (const ReqPtr &r : frozen) {
        r->parts.clear();
        r->parts.shrink_to_fit();
        finish(r, e);
    }
    return e;
}

// A device error ends every admitted and queued request.
void psf_engine::fail_all(int rc)
{
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
}

void psf_engine::run()
{
    std::vector<ReqPtr> picked, frozen;
    std::vector<int32_t> clear_b, clear_s;
    while (!stop.load()) {
        // The device is idle here.  Free the slots retired during the last
        // chunk, then place the requests picked meanwhile (or pick now).
        int rc = PSF_OK;
        if (!clear_b.empty()) {
            rc = psf_batch_clear_instances(batch, (int32_t)clear_b.size(), clear_b.data(), clear_s.data());
            clear_b.clear();
            clear_s.clear();
        }
        if (rc == PSF_OK && picked.empty()) {
            picked = pick();
            rc = stage(picked);
        }
        if (rc == PSF_OK) rc = place(picked);
        picked.clear();
        std::vector<ReqPtr> running;
        if (rc == PSF_OK) {
            std::lock_guard<std::mutex> lock(mu);
            for (auto &per : active)
                for (auto &r : per)
                    if (r && r->remaining > 0) running.push_back(r);
        }
        if (rc == PSF_OK && running.empty()) {
            if (!frozen.empty()) {
                rc = retire(frozen, clear_b, clear_s);
                frozen.clear();
                if (rc == PSF_OK) continue;
            } else {
                std::unique_lock<std::mutex> lock(mu);
                cv_work.wait_for(lock, std::chrono::milliseconds(20), [&] { return stop.load() || !queue.empty(); });
                continue;
            }
        }
        // Launch the next chunk; the rollouts that reach their step count in
        // it are retired during the chunk after it.
        int k = 0;
        const double ts = now();
        std::vector<ReqPtr> finishing;
        if (rc == PSF_OK) {
            int64_t most = 0;
            for (const ReqPtr &r : running) most = std::max(most, r->remaining);
            k = (int)std::min<int64_t>(chunk, most);
            rc = psf_batch_step(batch, k);
        }
        if (rc == PSF_OK) {
            for (const ReqPtr &r : running)
                if (r->remaining <= k) finishing.push_back(r);
            rc = retire(frozen, clear_b, clear_s);
            frozen.clear();
        }
        if (rc == PSF_OK) {
            picked = pick();
            rc = stage(picked);
        }
        if (rc == PSF_OK) rc = psf_batch_sync(batch);
        if (rc == PSF_OK) {
            std::lock_guard<std::mutex> lock(mu);
            st.step_launches += k;
            st.step_s += now() - ts;
            for (const ReqPtr &r : running) {
                const int64_t d = std::min<int64_t>(k, r->remaining);
                r->remaining -= d;
                st.instance_steps += d;
                st.particle_steps += d * ((int64_t)r->parts.size() / 4);
            }
            frozen = std::move(finishing);
        }
        if (rc != PSF_OK) {
            fail_all(rc);
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
    // Pinned staging for placements (two halves of up to four full-size
    // requests each), the reads beside a running chunk, and their events.
    e->arena_floats = 4 * std::max<int64_t>(cfg->max_particles, 1 << 12) * 4;
    cudaError_t ce = cudaSetDevice(device);
    if (ce == cudaSuccess)
        ce = cudaHostAlloc((void **)&e->arena, (size_t)(2 * e->arena_floats) * sizeof(float),
                           cudaHostAllocPortable);
    for (int h = 0; h < 2 && ce == cudaSuccess; ++h)
        ce = cudaEventCreateWithFlags(&e->half_done[h], cudaEventDisableTiming);
    rc = ce != cudaSuccess ? psf::cuda_fail(ce, "engine staging") : psf::batch_prepare_reads(e->batch);
    if (rc != PSF_OK) {
        e->release();
        delete e;
        return rc;
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
        e->release();
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
    e->release();
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
