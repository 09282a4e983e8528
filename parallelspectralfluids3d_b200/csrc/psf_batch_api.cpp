// C ABI of include/psf_batch.h: the batched engine.
//
// A batch owns, per basis, the BF16 hi/lo copies of C and Phi laid out for
// TMA (K-major rows of 64 elements, 128-byte swizzle), the slots' FP64 state
// and forcing, the BF16 hi/lo copy of the state used as the GEMMs' narrow
// operand, the partial sums of the contraction, the slots' face fields and
// particles; plus device tables of slots and of the slots' particle counts, so that one
// captured CUDA graph serves every occupancy of the slots.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "psf_b200.h"
#include "psf_batch.h"
#include "psf_batch_internal.h"
#include "psf_internal.h"

using psf::fail;

namespace {

inline int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

#define PSF_CHECK(x)                   \
    do {                               \
        int rc_ = (x);                 \
        if (rc_ != PSF_OK) return rc_; \
    } while (0)
#define PSF_CUDA(x)                                           \
    do {                                                      \
        cudaError_t e_ = (x);                                 \
        if (e_ != cudaSuccess) return psf::cuda_fail(e_, #x); \
    } while (0)

struct HostGroup {
    int N = 0, Nj = 0, Na = 0, a_tiles = 0;
    int cap = 0, bn = 0, slot_base = 0;
    int parts = 4;  // contraction partials per mode (a-tiles x K splits x 4 warps)
    int64_t F_act = 0, Fp = 0, n_faces = 0, pmax = 0;
    psf_grid grid{};
    std::vector<int8_t> sigma;
    uint16_t *C = nullptr;    // BF16 [N][2][Na][Nj]
    uint16_t *Phi = nullptr;  // BF16 [2][Fp][Nj]
    uint16_t *W = nullptr;    // BF16 [2][bn][Nj]
    double *lam = nullptr, *w = nullptr, *force = nullptr, *dwpart = nullptr;
    float *wf = nullptr;
    float2 *pairs = nullptr;
    std::vector<int32_t> faces_host, dst_host;  // for reading a slot's face field back
    int32_t *pair_dst = nullptr;
    int64_t V = 0;
    CUtensorMap mapC{}, mapPhi{}, mapW{};
};

// First-fit allocator of particle ranges in the batch's device pool, in
// units of 256 particles.
class RangePool {
public:
    void reset(int64_t units)
    {
        free_.clear();
        total_ = units;
        if (units > 0) free_[0] = units;
    }
    bool alloc(int64_t units, int64_t *start)
    {
        if (units == 0) {
            *start = 0;
            return true;
        }
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= units) {
                *start = it->first;
                const int64_t rest = it->second - units, at = it->first + units;
                free_.erase(it);
                if (rest > 0) free_[at] = rest;
                return true;
            }
        return false;
    }
    void release(int64_t start, int64_t units)
    {
        if (units == 0) return;
        auto it = free_.emplace(start, units).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    int64_t free_units() const
    {
        int64_t n = 0;
        for (const auto &r : free_) n += r.second;
        return n;
    }
    int64_t largest() const
    {
        int64_t n = 0;
        for (const auto &r : free_) n = std::max(n, r.second);
        return n;
    }

private:
    std::map<int64_t, int64_t> free_;
    int64_t total_ = 0;
};

}  // namespace

struct psf_batch {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<HostGroup> groups;
    std::vector<psf::SlotDev> slots;  // host mirror of the slot table
    std::vector<long long> prefix;  // host copy of the tracer's slot prefix sums
    psf::GroupDev *d_groups = nullptr;
    psf::SlotDev *d_slots = nullptr;
    long long *d_prefix = nullptr;
    int *d_err = nullptr;
    psf::StepArgs contract{};   // contraction units only
    psf::StepArgs recon{};      // reconstruction units only
    psf::StepArgs fused{};      // contraction, state update, reconstruction in one cooperative launch
    bool use_fused = true;
    unsigned int *grid_bar = nullptr;
    int bn_max = 64;
    int ksplit = 1;   // K ranges per contraction row tile
    int gemm_ctas = 148;
    int trace_ctas = 592;
    double tuned_ms = 0.0;
    psf::OrderBufs order{};
    int64_t pmax_all = 0;
    float4 *pool_parts = nullptr;   // particle pool shared by all slots
    int32_t *pool_perm = nullptr;
    int64_t pool_cap = 0;           // particles
    RangePool pool;
    std::vector<int64_t> slot_units;  // pool units held by each slot
    int64_t bytes = 0;
    std::vector<void *> allocs;
    // Reads of slots that the queued steps do not touch (psf::batch_read_frozen):
    // a second stream and pinned host buffers for one slot's particles.
    cudaStream_t side = nullptr;
    float4 *rd_parts = nullptr;
    int32_t *rd_perm = nullptr;
    int64_t rd_cap = 0;
    // Host rows read by copies queued without a synchronisation.
    std::vector<std::vector<double>> kept_rows;

    ~psf_batch()
    {
        drop_graph();
        for (void *p : allocs) cudaFree(p);
        if (rd_parts) cudaFreeHost(rd_parts);
        if (rd_perm) cudaFreeHost(rd_perm);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }
    void drop_graph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    template <class T>
    int alloc(T **p, size_t count)
    {
        void *v = nullptr;
        const size_t n = std::max<size_t>(1, count) * sizeof(T);
        cudaError_t e = cudaMalloc(&v, n);
        if (e != cudaSuccess) return psf::cuda_fail(e, "cudaMalloc");
        allocs.push_back(v);
        bytes += (int64_t)n;
        *p = static_cast<T *>(v);
        return PSF_OK;
    }
    int n_slots() const { return (int)slots.size(); }
};

namespace {

int upload_basis(psf_batch *B, HostGroup &G, const psf_batch_basis &bb)
{
    const psf_basis_desc &b = bb.basis;
    const int N = G.N;
    cudaStream_t st = B->stream;
    // C as BF16 hi/lo [k][hl][a][j], a padded to Na and j to Nj with zeros.
    {
        std::vector<uint16_t> h((size_t)N * 2 * G.Na * G.Nj, 0);
        for (int k = 0; k < N; ++k)
            for (int a = 0; a < N; ++a) {
                const double *src = b.advection + ((size_t)k * N + a) * N;
                uint16_t *hi = h.data() + (((size_t)k * 2 + 0) * G.Na + a) * G.Nj;
                uint16_t *lo = h.data() + (((size_t)k * 2 + 1) * G.Na + a) * G.Nj;
                for (int j = 0; j < N; ++j) psf::split_bf16_host(src[j], hi + j, lo + j);
            }
        PSF_CHECK(B->alloc(&G.C, h.size()));
        PSF_CUDA(cudaMemcpyAsync(G.C, h.data(), h.size() * 2, cudaMemcpyHostToDevice, st));
        PSF_CUDA(cudaStreamSynchronize(st));
    }
    // Phi (tracer signs folded in) as BF16 hi/lo [hl][f][i], f padded to Fp.
    {
        std::vector<uint16_t> h((size_t)2 * G.Fp * G.Nj, 0);
        for (int64_t r = 0; r < G.F_act; ++r) {
            const double s = (double)G.sigma[(size_t)b.active_faces[r]];
            uint16_t *hi = h.data() + ((size_t)0 * G.Fp + r) * G.Nj;
            uint16_t *lo = h.data() + ((size_t)1 * G.Fp + r) * G.Nj;
            for (int i = 0; i < N; ++i) psf::split_bf16_host(s * b.phi[(size_t)r * N + i], hi + i, lo + i);
        }
        PSF_CHECK(B->alloc(&G.Phi, h.size()));
        PSF_CUDA(cudaMemcpyAsync(G.Phi, h.data(), h.size() * 2, cudaMemcpyHostToDevice, st));
        PSF_CUDA(cudaStreamSynchronize(st));
    }
    PSF_CHECK(B->alloc(&G.lam, (size_t)N));
    PSF_CUDA(cudaMemcpyAsync(G.lam, b.eigenvalues, (size_t)N * 8, cudaMemcpyHostToDevice, st));

    const size_t cap = (size_t)G.cap;
    PSF_CHECK(B->alloc(&G.W, (size_t)2 * G.bn * G.Nj));
    PSF_CHECK(B->alloc(&G.w, cap * N));
    PSF_CHECK(B->alloc(&G.wf, cap * N));
    PSF_CUDA(cudaMemsetAsync(G.wf, 0, cap * N * 4, st));
    PSF_CHECK(B->alloc(&G.force, cap * N));
    PSF_CHECK(B->alloc(&G.dwpart, (size_t)N * G.a_tiles * 4 * psf::GEMM_MAX_KSPLIT * cap));
    G.faces_host.assign(b.active_faces, b.active_faces + G.F_act);
    psf::face_pair_slots(G.grid, b.active_faces, G.F_act, G.dst_host);
    PSF_CHECK(B->alloc(&G.pair_dst, G.dst_host.size()));
    PSF_CUDA(cudaMemcpyAsync(G.pair_dst, G.dst_host.data(), G.dst_host.size() * 4, cudaMemcpyHostToDevice, st));
    PSF_CUDA(cudaStreamSynchronize(st));
    PSF_CHECK(B->alloc(&G.pairs, cap * (size_t)(3 * G.V)));
    PSF_CUDA(cudaMemsetAsync(G.pairs, 0, cap * (size_t)(3 * G.V) * sizeof(float2), st));
    PSF_CUDA(cudaMemsetAsync(G.W, 0, (size_t)2 * G.bn * G.Nj * 2, st));
    PSF_CUDA(cudaMemsetAsync(G.w, 0, cap * N * 8, st));
    PSF_CUDA(cudaMemsetAsync(G.force, 0, cap * N * 8, st));
    PSF_CUDA(cudaMemsetAsync(G.dwpart, 0, (size_t)N * G.a_tiles * 4 * psf::GEMM_MAX_KSPLIT * cap * 8, st));

    // Tensor maps: inner dimension first, strides in bytes for dims 1..
    {
        const uint64_t dims[4] = {(uint64_t)G.Nj, (uint64_t)G.Na, 2, (uint64_t)N};
        const uint64_t str[3] = {(uint64_t)G.Nj * 2, (uint64_t)G.Na * G.Nj * 2, (uint64_t)2 * G.Na * G.Nj * 2};
        const uint32_t box[4] = {64, 128, 2, 1};
        PSF_CHECK(psf::encode_tensor_map(&G.mapC, G.C, 4, dims, str, box));
    }
    {
        const uint64_t dims[4] = {(uint64_t)G.Nj, (uint64_t)G.Fp, 2, 1};
        const uint64_t str[3] = {(uint64_t)G.Nj * 2, (uint64_t)G.Fp * G.Nj * 2, (uint64_t)2 * G.Fp * G.Nj * 2};
        const uint32_t box[4] = {64, 128, 2, 1};
        PSF_CHECK(psf::encode_tensor_map(&G.mapPhi, G.Phi, 4, dims, str, box));
    }
    {
        const uint64_t dims[3] = {(uint64_t)G.Nj, (uint64_t)G.bn, 2};
        const uint64_t str[2] = {(uint64_t)G.Nj * 2, (uint64_t)G.bn * G.Nj * 2};
        const uint32_t box[3] = {64, (uint32_t)G.bn, 2};
        PSF_CHECK(psf::encode_tensor_map(&G.mapW, G.W, 3, dims, str, box));
    }
    return PSF_OK;
}

void fill_gemm_args(psf_batch *B)
{
    psf::StepArgs &c = B->contract;
    psf::StepArgs &r = B->recon;
    std::memset(&c, 0, sizeof(c));
    const int n = (int)B->groups.size();
    c.n_groups = n;
    c.err = B->d_err;
    c.grid_bar = B->grid_bar;
    c.groups = B->d_groups;
    c.slots = B->d_slots;
    c.n_slots = B->n_slots();
    for (int gi = 0; gi < n; ++gi) {
        HostGroup &G = B->groups[(size_t)gi];
        const uint32_t tx = 2u * 128u * 128u + 2u * (uint32_t)G.bn * 128u;
        psf::GemmGroup &x = c.g[gi];
        x.tmA = G.mapC;
        x.tmB = G.mapW;
        x.m_inner = G.a_tiles;
        x.k_chunks = G.Nj / 64;
        x.ksplit = std::max(1, std::min(B->ksplit, x.k_chunks));
        x.kc_per = (x.k_chunks + x.ksplit - 1) / x.ksplit;
        x.ksplit = (x.k_chunks + x.kc_per - 1) / x.kc_per;  // no empty K range
        x.tiles = G.N * G.a_tiles * x.ksplit;
        G.parts = G.a_tiles * x.ksplit * 4;
        x.nparts = G.parts;
        x.bn = G.bn;
        x.tx_bytes = tx;
        x.cap = G.cap;
        x.n_rows = G.N;
        x.ldw = G.N;
        x.wf = G.wf;
        x.dwpart = G.dwpart;
        c.c_tiles += x.tiles;
        psf::GemmGroup &y = c.g[n + gi];
        y.tmA = G.mapPhi;
        y.tmB = G.mapW;
        y.tiles = (int)(G.Fp / 128);
        y.m_inner = y.tiles;
        y.k_chunks = G.Nj / 64;
        y.ksplit = 1;
        y.kc_per = y.k_chunks;
        y.bn = G.bn;
        y.tx_bytes = tx;
        y.cap = G.cap;
        y.n_rows = (int)G.F_act;
        y.ldw = G.N;
        y.n_faces = G.n_faces;
        y.pair_dst = G.pair_dst;
        y.pairs = reinterpret_cast<float *>(G.pairs);
        y.pair_floats = 6 * G.V;
        y.slot_of = B->d_slots + G.slot_base;
        c.r_tiles += y.tiles;
    }
    B->fused = c;
    B->fused.fused = 1;
    r = c;
    r.c_tiles = 0;     // reconstruction units only
    c.r_tiles = 0;     // contraction units only
}

int upload_tables(psf_batch *B)
{
    std::vector<psf::GroupDev> gd(B->groups.size());
    for (size_t gi = 0; gi < B->groups.size(); ++gi) {
        const HostGroup &G = B->groups[gi];
        psf::GroupDev &d = gd[gi];
        d.grid = psf::make_grid_dev(G.grid);
        d.N = G.N;
        d.Nj = G.Nj;
        d.cap = G.cap;
        d.bn = G.bn;
        d.a_tiles = G.a_tiles;
        d.nparts = G.parts;
        d.slot_base = G.slot_base;
        d.n_faces = G.n_faces;
        d.pmax = G.pmax;
        d.w = G.w;
        d.wf = G.wf;
        d.force = G.force;
        d.lam = G.lam;
        d.dwpart = G.dwpart;
        d.W = G.W;
        d.pairs = G.pairs;
        d.V = G.V;
        d.parts = B->pool_parts;
        d.perm = B->pool_perm;
    }
    PSF_CUDA(cudaMemcpyAsync(B->d_groups, gd.data(), gd.size() * sizeof(psf::GroupDev), cudaMemcpyHostToDevice,
                             B->stream));
    PSF_CUDA(cudaMemcpyAsync(B->d_slots, B->slots.data(), B->slots.size() * sizeof(psf::SlotDev),
                             cudaMemcpyHostToDevice, B->stream));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    return PSF_OK;
}

int upload_prefix(psf_batch *B)
{
    const size_t n = B->slots.size();
    B->prefix.assign(n + 1, 0);
    for (size_t s = 0; s < n; ++s)
        B->prefix[s + 1] = B->prefix[s] + (B->slots[s].active ? B->slots[s].n_particles : 0);
    PSF_CUDA(cudaMemcpyAsync(B->d_prefix, B->prefix.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice,
                             B->stream));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    return PSF_OK;
}

int check_device_error(psf_batch *B)
{
    int code = 0;
    PSF_CUDA(cudaMemcpyAsync(&code, B->d_err, sizeof(int), cudaMemcpyDeviceToHost, B->stream));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    if (code != 0) return fail(PSF_ERR_TIMEOUT, "a tensor-core kernel gave up a bounded wait (code " +
                                                    std::to_string(code) + "); destroy the batch");
    return PSF_OK;
}

int fused_grid(psf_batch *B)
{
    return std::max(1, std::min(B->gemm_ctas, psf::max_fused_grid(B->bn_max, B->num_sms)));
}

// The tensor-core part of a step: one cooperative launch (fused), or the
// contraction, the state kernel and the reconstruction as three launches.
int launch_tc_part(psf_batch *B, cudaStream_t st, bool fused)
{
    if (fused) {
        PSF_CUDA(cudaMemsetAsync(B->grid_bar, 0, sizeof(unsigned int), st));
        return psf::launch_batch_step_tc(B->fused, B->bn_max, fused_grid(B), st);
    }
    PSF_CHECK(psf::launch_batch_step_tc(B->contract, B->bn_max, B->gemm_ctas, st));
    PSF_CHECK(psf::launch_batch_state(B->d_groups, B->d_slots, B->n_slots(), st));
    PSF_CHECK(psf::launch_batch_step_tc(B->recon, B->bn_max, B->gemm_ctas, st));
    return PSF_OK;
}

// Project-written autotuner: time every kernel variant that fits the batch
// (MMA columns 64 / 128 / 256, i.e. 4 / 3 / 2 pipeline stages; persistent
// grids of 1x and 1/2x the SM count; 1, 2 or 4 K ranges per contraction row
// tile) on the tensor-core part of a step exactly as the step will run it
// (one fused launch, or three launches), and keep the fastest.  Run at
// creation, when every slot is empty, so the timed launches change nothing.
//
// The fused launch is cooperative: it starts only when the previous step's
// tracer has left every SM, so in a step it costs more than when timed back
// to back.  Measured on three workloads (64 slots of N=128 and of N=384, 512
// slots of uneven N), a step with the fused launch took 6-13 us more than its
// tensor-core time difference predicts; the fused candidates are charged
// FUSED_STEP_PENALTY_MS for it.
constexpr double FUSED_STEP_PENALTY_MS = 0.010;

int autotune(psf_batch *B, int need_bn)
{
    const int variants[3] = {64, 128, 256};
    const int grids[2] = {B->num_sms, std::max(1, B->num_sms / 2)};
    const int splits[3] = {1, 2, 4};
    const bool try_fused = B->use_fused;  // a batch created unfused stays unfused
    cudaEvent_t e0, e1;
    PSF_CUDA(cudaEventCreate(&e0));
    PSF_CUDA(cudaEventCreate(&e1));
    double best = 1e30, best_ms = 0.0;
    int best_bn = -1, best_grid = B->num_sms, best_ks = 1;
    int rc = PSF_OK;
    bool best_fused = try_fused;
    // Time the launches as full slots would run them: the reconstruction
    // writes face pairs only for slots marked as stepped.
    for (psf::SlotDev &s : B->slots) s.stepped = 1;
    for (int fu = try_fused ? 1 : 0; fu >= 0; --fu)
    for (int v : variants) {
        if (v < need_bn) continue;
        for (int g : grids) {
            for (int ks : splits) {
                B->use_fused = fu == 1;
                B->bn_max = v;
                B->gemm_ctas = g;
                B->ksplit = ks;
                fill_gemm_args(B);
                if ((rc = upload_tables(B)) != PSF_OK) break;
                for (int rep = 0; rc == PSF_OK && rep < 2; ++rep) rc = launch_tc_part(B, B->stream, B->use_fused);
                const int reps = 5;
                cudaEventRecord(e0, B->stream);
                for (int rep = 0; rc == PSF_OK && rep < reps; ++rep) rc = launch_tc_part(B, B->stream, B->use_fused);
                cudaEventRecord(e1, B->stream);
                cudaError_t e = cudaEventSynchronize(e1);
                if (rc == PSF_OK && e != cudaSuccess) rc = psf::cuda_fail(e, "autotune");
                if (rc == PSF_OK) rc = check_device_error(B);
                if (rc != PSF_OK) break;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                const double cost = ms / reps + (B->use_fused ? FUSED_STEP_PENALTY_MS : 0.0);
                if (cost < best) {
                    best = cost;
                    best_ms = ms / reps;
                    best_bn = v;
                    best_grid = g;
                    best_ks = ks;
                    best_fused = B->use_fused;
                }
            }
            if (rc != PSF_OK) break;
        }
        if (rc != PSF_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (psf::SlotDev &s : B->slots) s.stepped = 0;
    if (rc != PSF_OK) {
        upload_tables(B);
        return rc;
    }
    B->bn_max = best_bn;
    B->gemm_ctas = best_grid;
    B->ksplit = best_ks;
    B->use_fused = best_fused;
    B->tuned_ms = best_ms;
    fill_gemm_args(B);
    return upload_tables(B);
}

int launch_step(psf_batch *B, cudaStream_t st)
{
    PSF_CHECK(launch_tc_part(B, st, B->use_fused));
    PSF_CHECK(psf::launch_batch_trace(B->d_groups, B->d_slots, B->d_prefix, B->n_slots(), B->trace_ctas, st));
    return PSF_OK;
}

int build_graph(psf_batch *B)
{
    if (B->exec) return PSF_OK;
    PSF_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    int rc = launch_step(B, B->stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(B->stream, &g);
    if (rc != PSF_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return psf::cuda_fail(e, "cudaStreamEndCapture");
    B->graph = g;
    PSF_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
    return PSF_OK;
}

int slot_index(psf_batch *B, int32_t basis, int32_t slot, int *sg)
{
    if (!B) return fail(PSF_ERR_INVALID, "null batch");
    if (basis < 0 || basis >= (int)B->groups.size()) return fail(PSF_ERR_INVALID, "basis index out of range");
    if (slot < 0 || slot >= B->groups[(size_t)basis].cap) return fail(PSF_ERR_INVALID, "slot index out of range");
    *sg = B->groups[(size_t)basis].slot_base + slot;
    return PSF_OK;
}

psf::PlainDev particle_view(psf_batch *B, int basis, int slot, int64_t count)
{
    HostGroup &G = B->groups[(size_t)basis];
    const psf::SlotDev &s = B->slots[(size_t)(G.slot_base + slot)];
    psf::PlainDev d{};
    d.grid = psf::make_grid_dev(G.grid);
    d.P = count;
    d.parts = B->pool_parts + s.poff;
    d.perm = B->pool_perm + s.poff;
    return d;
}

}  // namespace

extern "C" {

int psf_batch_create(const psf_batch_config *cfg, int device, psf_batch **out)
{
    if (!cfg || !out || !cfg->bases) return fail(PSF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->n_bases < 1 || cfg->n_bases > PSF_BATCH_MAX_BASES)
        return fail(PSF_ERR_UNSUPPORTED, "n_bases must be in [1, PSF_BATCH_MAX_BASES]");
    if (cfg->precision != PSF_PRECISION_BF16X2)
        return fail(PSF_ERR_UNSUPPORTED, "batches run the BF16 hi/lo tensor-core path (PSF_PRECISION_BF16X2)");
    if (cfg->gemm_columns != 0 && cfg->gemm_columns != 64 && cfg->gemm_columns != 128 && cfg->gemm_columns != 256)
        return fail(PSF_ERR_INVALID, "gemm_columns must be 0, 64, 128 or 256");
    int need_bn = 16;
    for (int i = 0; i < cfg->n_bases; ++i) {
        const psf_batch_basis &bb = cfg->bases[i];
        const psf_basis_desc &b = bb.basis;
        if (bb.slots < 1 || bb.slots > PSF_BATCH_MAX_SLOTS)
            return fail(PSF_ERR_UNSUPPORTED, "slots per basis must be in [1, PSF_BATCH_MAX_SLOTS]");
        if (bb.max_particles < 0 || bb.max_particles > INT32_MAX)
            return fail(PSF_ERR_INVALID, "max_particles out of range");
        if (b.n_modes < 1 || b.n_modes > psf::PSF_MAX_MODES)
            return fail(PSF_ERR_UNSUPPORTED, "n_modes must be in [1, 1024]");
        if (b.n_active < 1 || !b.active_faces || !b.phi || !b.advection || !b.eigenvalues || !b.sign_bits)
            return fail(PSF_ERR_INVALID, "basis arrays must not be null");
        if (b.grid.dims[0] == 0 || b.grid.dims[1] == 0 || b.grid.dims[2] == 0 || !(b.grid.resolution > 0.0))
            return fail(PSF_ERR_INVALID, "grid dims and resolution must be positive");
        if (b.grid.dims[0] > 1023 || b.grid.dims[1] > 1023 || b.grid.dims[2] > 1023)
            return fail(PSF_ERR_UNSUPPORTED, "grid dims above 1023 voxels per axis");
        const int64_t F = psf::n_faces_of(b.grid);
        const int64_t V = (int64_t)b.grid.dims[0] * b.grid.dims[1] * b.grid.dims[2];
        if (F >= (int64_t)INT32_MAX || 6 * V >= (int64_t)INT32_MAX)
            return fail(PSF_ERR_UNSUPPORTED, "grid has too many faces");
        for (int64_t r = 0; r < b.n_active; ++r)
            if (b.active_faces[r] < 0 || b.active_faces[r] >= F)
                return fail(PSF_ERR_INVALID, "active face id out of range");
        need_bn = std::max(need_bn, (int)round_up(bb.slots, 16));
    }
    if (cfg->contraction_ksplit != 0 && cfg->contraction_ksplit != 1 && cfg->contraction_ksplit != 2 &&
        cfg->contraction_ksplit != 4)
        return fail(PSF_ERR_INVALID, "contraction_ksplit must be 0, 1, 2 or 4");
    if (cfg->gemm_columns != 0 && cfg->gemm_columns < need_bn)
        return fail(PSF_ERR_INVALID, "gemm_columns is smaller than the slots of a basis");

    psf_batch *B = nullptr;
    try {
        B = new psf_batch();
    } catch (const std::bad_alloc &) {
        return fail(PSF_ERR_NOMEM, "host allocation failed");
    }
    auto bail = [&](int rc) {
        delete B;
        return rc;
    };
    B->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(psf::cuda_fail(e, "cudaSetDevice"));
    cudaDeviceGetAttribute(&B->num_sms, cudaDevAttrMultiProcessorCount, device);
    e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(psf::cuda_fail(e, "cudaStreamCreate"));
    int rc = PSF_OK;
    if ((rc = B->alloc(&B->d_err, 1)) != PSF_OK || (rc = B->alloc(&B->grid_bar, 1)) != PSF_OK) return bail(rc);
    B->use_fused = cfg->unfused == 0;
    if ((e = cudaMemsetAsync(B->d_err, 0, sizeof(int), B->stream)) != cudaSuccess)
        return bail(psf::cuda_fail(e, "cudaMemset"));

    int slot_base = 0;
    B->groups.resize((size_t)cfg->n_bases);
    try {
        for (int i = 0; i < cfg->n_bases; ++i) {
            const psf_batch_basis &bb = cfg->bases[i];
            HostGroup &G = B->groups[(size_t)i];
            G.N = bb.basis.n_modes;
            G.Nj = (int)round_up(G.N, 64);
            G.Na = (int)round_up(G.N, 128);
            G.a_tiles = G.Na / 128;
            G.cap = bb.slots;
            G.bn = (int)round_up(bb.slots, 16);
            G.slot_base = slot_base;
            G.F_act = bb.basis.n_active;
            G.Fp = round_up(G.F_act, 128);
            G.grid = bb.basis.grid;
            G.n_faces = psf::n_faces_of(G.grid);
            G.V = (int64_t)G.grid.dims[0] * G.grid.dims[1] * G.grid.dims[2];
            G.pmax = round_up(std::max<int64_t>(1, bb.max_particles), 256);
            B->pmax_all = std::max(B->pmax_all, G.pmax);
            slot_base += G.cap;
            if ((rc = psf::fold_signs(G.grid, bb.basis.sign_bits, G.sigma)) != PSF_OK) return bail(rc);
            if ((rc = upload_basis(B, G, bb)) != PSF_OK) return bail(rc);
        }
        B->slots.assign((size_t)slot_base, psf::SlotDev{});
        for (const HostGroup &G : B->groups)
            for (int b = 0; b < G.cap; ++b) {
                psf::SlotDev &s = B->slots[(size_t)(G.slot_base + b)];
                s.group = (int)(&G - B->groups.data());
                s.slot = b;
            }
    } catch (const std::bad_alloc &) {
        return bail(fail(PSF_ERR_NOMEM, "host staging allocation failed"));
    }
    {
        int64_t all_slots = 0;
        for (const HostGroup &G : B->groups) all_slots += (int64_t)G.cap * G.pmax;
        B->pool_cap = cfg->particle_pool > 0 ? round_up(cfg->particle_pool, 256) : all_slots;
        if (B->pool_cap > (int64_t)INT32_MAX) return bail(fail(PSF_ERR_UNSUPPORTED, "particle pool too large"));
        B->pool.reset(B->pool_cap / 256);
        B->slot_units.assign((size_t)slot_base, 0);
    }
    if ((rc = B->alloc(&B->pool_parts, (size_t)B->pool_cap)) || (rc = B->alloc(&B->pool_perm, (size_t)B->pool_cap)) ||
        (rc = B->alloc(&B->d_groups, B->groups.size())) || (rc = B->alloc(&B->d_slots, B->slots.size())) ||
        (rc = B->alloc(&B->d_prefix, B->slots.size() + 1)))
        return bail(rc);
    // Particle ordering scratch, sized for the largest slot.
    {
        psf::OrderBufs &o = B->order;
        size_t tmp = 0;
        unsigned char *temp = nullptr;
        if ((rc = psf::sort_particles_temp_bytes(B->pmax_all, &tmp)) || (rc = B->alloc(&o.staging, B->pmax_all)) ||
            (rc = B->alloc(&o.keys_in, B->pmax_all)) || (rc = B->alloc(&o.keys_out, B->pmax_all)) ||
            (rc = B->alloc(&o.idx_in, B->pmax_all)) || (rc = B->alloc(&temp, tmp)))
            return bail(rc);
        o.temp = temp;
        o.temp_bytes = tmp;
    }
    fill_gemm_args(B);
    if ((rc = upload_tables(B)) != PSF_OK || (rc = upload_prefix(B)) != PSF_OK) return bail(rc);
    B->trace_ctas = psf::batch_trace_grid(B->num_sms);
    B->gemm_ctas = cfg->gemm_ctas > 0 ? cfg->gemm_ctas : B->num_sms;
    if (cfg->gemm_columns != 0) {
        B->bn_max = cfg->gemm_columns;
    } else if (cfg->autotune) {
        if ((rc = autotune(B, need_bn)) != PSF_OK) return bail(rc);
        if (cfg->gemm_ctas > 0) B->gemm_ctas = cfg->gemm_ctas;
    } else {
        B->bn_max = need_bn <= 64 ? 64 : (need_bn <= 128 ? 128 : 256);
    }
    if (cfg->contraction_ksplit > 0) {
        B->ksplit = cfg->contraction_ksplit;
        fill_gemm_args(B);
        if ((rc = upload_tables(B)) != PSF_OK) return bail(rc);
    }
    *out = B;
    return PSF_OK;
}

int psf_batch_destroy(psf_batch *B)
{
    if (!B) return PSF_OK;
    cudaSetDevice(B->device);
    if (B->stream) cudaStreamSynchronize(B->stream);
    delete B;
    return PSF_OK;
}

int psf_batch_info_get(psf_batch *B, psf_batch_info *info)
{
    if (!B || !info) return fail(PSF_ERR_INVALID, "null argument");
    info->gemm_columns = B->bn_max;
    info->gemm_ctas = B->gemm_ctas;
    info->trace_ctas = B->trace_ctas;
    info->kernels_per_step = B->use_fused ? 2 : 4;
    info->device_bytes = B->bytes;
    info->tuned_ms = B->tuned_ms;
    info->contraction_ksplit = B->ksplit;
    return PSF_OK;
}

}  // extern "C"

namespace {

// Place one instance without finishing the slot tables: the caller uploads
// the prefix sums, primes the contraction and synchronises once for a group
// of placements.  Host rows given to the asynchronous copies are kept in
// `keep` until then.
int set_one(psf_batch *B, int32_t basis, int32_t slot, const psf_instance_desc *inst,
            std::vector<std::vector<double>> &keep)
{
    int sg = 0;
    PSF_CHECK(slot_index(B, basis, slot, &sg));
    if (!inst || !inst->w0) return fail(PSF_ERR_INVALID, "null argument");
    HostGroup &G = B->groups[(size_t)basis];
    const psf_params &p = inst->params;
    if (inst->n_modes < 1 || inst->n_modes > G.N)
        return fail(PSF_ERR_INVALID, "n_modes must be in [1, the basis' n_modes]");
    if (inst->n_particles < 0 || inst->n_particles > G.pmax)
        return fail(PSF_ERR_INVALID, "n_particles exceeds the slot's capacity");
    if (inst->n_particles > 0 && !inst->particles) return fail(PSF_ERR_INVALID, "particles is null");
    if (!(p.timestep > 0.0) || !std::isfinite(p.timestep))
        return fail(PSF_ERR_INVALID, "timestep must be positive and finite");
    if (p.integrator != PSF_RK1 && p.integrator != PSF_RK4)
        return fail(PSF_ERR_INVALID, "integrator must be PSF_RK1 or PSF_RK4");
    if ((p.flags & PSF_FLAG_FORCING) && !inst->forcing)
        return fail(PSF_ERR_INVALID, "PSF_FLAG_FORCING is set but forcing is null");
    if (inst->steps < 0) return fail(PSF_ERR_INVALID, "steps must be >= 0");
    cudaStream_t st = B->stream;
    // Particle range: give back the slot's old one, then take a new one.
    psf::SlotDev &s = B->slots[(size_t)sg];
    if (B->slot_units[(size_t)sg] > 0) {
        PSF_CUDA(cudaStreamSynchronize(st));
        B->pool.release(s.poff / 256, B->slot_units[(size_t)sg]);
        B->slot_units[(size_t)sg] = 0;
    }
    const int64_t units = (inst->n_particles + 255) / 256;
    int64_t start = 0;
    if (!B->pool.alloc(units, &start)) {
        s.active = 0;
        s.n_particles = 0;
        PSF_CUDA(cudaMemcpyAsync(B->d_slots + sg, &s, sizeof(s), cudaMemcpyHostToDevice, st));
        return fail(PSF_ERR_NOMEM, "the particle pool has no free range for this instance");
    }
    B->slot_units[(size_t)sg] = units;
    keep.emplace_back((size_t)(2 * G.N), 0.0);
    std::vector<double> &rows = keep.back();
    std::memcpy(rows.data(), inst->w0, (size_t)inst->n_modes * 8);
    if (inst->forcing) std::memcpy(rows.data() + G.N, inst->forcing, (size_t)inst->n_modes * 8);
    PSF_CUDA(cudaMemcpyAsync(G.w + (size_t)slot * G.N, rows.data(), (size_t)G.N * 8, cudaMemcpyHostToDevice, st));
    PSF_CUDA(cudaMemcpyAsync(G.force + (size_t)slot * G.N, rows.data() + G.N, (size_t)G.N * 8,
                             cudaMemcpyHostToDevice, st));
    s.active = 1;
    s.poff = start * 256;
    s.target = (unsigned long long)inst->steps;
    s.stepped = 0;
    s.n_modes = inst->n_modes;
    s.rk4 = p.integrator == PSF_RK4;
    s.flags = p.flags;
    s.dt = p.timestep;
    s.visc_signed = (p.flags & PSF_FLAG_DECAY_NEG) ? -p.viscosity : p.viscosity;
    s.lifetime = p.lifetime;
    s.seed = p.seed;
    s.step = 0;
    s.n_particles = inst->n_particles;
    PSF_CUDA(cudaMemcpyAsync(B->d_slots + sg, &s, sizeof(s), cudaMemcpyHostToDevice, st));
    PSF_CHECK(psf::launch_batch_pack(B->d_groups, B->d_slots, sg, st));
    if (inst->n_particles > 0) {
        PSF_CUDA(cudaMemcpyAsync(B->order.staging, inst->particles, (size_t)inst->n_particles * 16,
                                 cudaMemcpyHostToDevice, st));
        PSF_CHECK(psf::launch_order_particles(particle_view(B, basis, slot, inst->n_particles), B->order, st));
    }
    return PSF_OK;
}

// After placements: new prefix sums, the contraction partials a fused step
// starts from, and (unless `sync` is false) one synchronisation.
int finish_placements(psf_batch *B, bool sync = true)
{
    PSF_CHECK(upload_prefix(B));
    if (B->use_fused) PSF_CHECK(psf::launch_batch_step_tc(B->contract, B->bn_max, B->gemm_ctas, B->stream));
    if (sync) {
        PSF_CUDA(cudaStreamSynchronize(B->stream));
        B->kept_rows.clear();
    }
    return PSF_OK;
}

}  // namespace

extern "C" {

int psf_batch_set_instance(psf_batch *B, int32_t basis, int32_t slot, const psf_instance_desc *inst)
{
    if (!B) return fail(PSF_ERR_INVALID, "null batch");
    PSF_CUDA(cudaSetDevice(B->device));
    std::vector<std::vector<double>> keep;
    const int rc = set_one(B, basis, slot, inst, keep);
    const std::string msg = psf::g_last_error;
    const int rc2 = finish_placements(B);
    if (rc != PSF_OK) return fail(rc, msg);
    return rc2;
}

int psf_batch_set_instances(psf_batch *B, int32_t n, const int32_t *basis, const int32_t *slot,
                            const psf_instance_desc *const *inst, int32_t *status)
{
    if (!B || n < 0 || (n > 0 && (!basis || !slot || !inst || !status))) return fail(PSF_ERR_INVALID, "null argument");
    PSF_CUDA(cudaSetDevice(B->device));
    std::vector<std::vector<double>> keep;
    for (int32_t i = 0; i < n; ++i) status[i] = set_one(B, basis[i], slot[i], inst[i], keep);
    return finish_placements(B);
}

int psf_batch_clear_instances(psf_batch *B, int32_t n, const int32_t *basis, const int32_t *slot)
{
    if (!B || n < 0 || (n > 0 && (!basis || !slot))) return fail(PSF_ERR_INVALID, "null argument");
    PSF_CUDA(cudaSetDevice(B->device));
    bool synced = false;
    for (int32_t i = 0; i < n; ++i) {
        int sg = 0;
        PSF_CHECK(slot_index(B, basis[i], slot[i], &sg));
        HostGroup &G = B->groups[(size_t)basis[i]];
        psf::SlotDev &s = B->slots[(size_t)sg];
        if (B->slot_units[(size_t)sg] > 0) {
            if (!synced) PSF_CUDA(cudaStreamSynchronize(B->stream));
            synced = true;
            B->pool.release(s.poff / 256, B->slot_units[(size_t)sg]);
            B->slot_units[(size_t)sg] = 0;
        }
        s.active = 0;
        s.n_particles = 0;
        s.stepped = 0;
        PSF_CUDA(cudaMemsetAsync(G.w + (size_t)slot[i] * G.N, 0, (size_t)G.N * 8, B->stream));
        PSF_CUDA(cudaMemcpyAsync(B->d_slots + sg, &s, sizeof(s), cudaMemcpyHostToDevice, B->stream));
        PSF_CHECK(psf::launch_batch_pack(B->d_groups, B->d_slots, sg, B->stream));
    }
    return upload_prefix(B);
}

int psf_batch_clear_instance(psf_batch *B, int32_t basis, int32_t slot)
{
    return psf_batch_clear_instances(B, 1, &basis, &slot);
}

int psf_batch_read_instances(psf_batch *B, int32_t n, const int32_t *basis, const int32_t *slot, double *const *w,
                             float *const *xyzw)
{
    if (!B || n < 0 || (n > 0 && (!basis || !slot || !w || !xyzw))) return fail(PSF_ERR_INVALID, "null argument");
    PSF_CUDA(cudaSetDevice(B->device));
    for (int32_t i = 0; i < n; ++i) {
        int sg = 0;
        PSF_CHECK(slot_index(B, basis[i], slot[i], &sg));
        const psf::SlotDev &s = B->slots[(size_t)sg];
        if (!s.active) return fail(PSF_ERR_STATE, "slot is empty");
        HostGroup &G = B->groups[(size_t)basis[i]];
        if (w[i])
            PSF_CUDA(cudaMemcpyAsync(w[i], G.w + (size_t)slot[i] * G.N, (size_t)s.n_modes * 8, cudaMemcpyDeviceToHost,
                                     B->stream));
        if (xyzw[i] && s.n_particles > 0) {
            // Scatter back to the caller's order in a per-slot region of the
            // ordering scratch is not possible for several slots at once, so
            // each slot is un-ordered into the staging buffer and copied.
            PSF_CHECK(psf::launch_unorder_particles(particle_view(B, basis[i], slot[i], s.n_particles), B->order,
                                                    B->stream));
            PSF_CUDA(cudaMemcpyAsync(xyzw[i], B->order.staging, (size_t)s.n_particles * 16, cudaMemcpyDeviceToHost,
                                     B->stream));
        }
    }
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    return check_device_error(B);
}

int psf_batch_pool_free(psf_batch *B, int64_t *free_particles, int64_t *largest_range)
{
    if (!B || !free_particles || !largest_range) return fail(PSF_ERR_INVALID, "null argument");
    *free_particles = B->pool.free_units() * 256;
    *largest_range = B->pool.largest() * 256;
    return PSF_OK;
}

int psf_batch_step(psf_batch *B, int32_t nsteps)
{
    if (!B) return fail(PSF_ERR_INVALID, "null batch");
    if (nsteps < 0) return fail(PSF_ERR_INVALID, "nsteps must be >= 0");
    PSF_CUDA(cudaSetDevice(B->device));
    PSF_CHECK(build_graph(B));
    for (int32_t i = 0; i < nsteps; ++i) PSF_CUDA(cudaGraphLaunch(B->exec, B->stream));
    return PSF_OK;
}

int psf_batch_sync(psf_batch *B)
{
    if (!B) return fail(PSF_ERR_INVALID, "null batch");
    PSF_CUDA(cudaSetDevice(B->device));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    B->kept_rows.clear();
    return check_device_error(B);
}

int psf_batch_get_stream(psf_batch *B, void **stream)
{
    if (!B || !stream) return fail(PSF_ERR_INVALID, "null argument");
    *stream = (void *)B->stream;
    return PSF_OK;
}

int psf_batch_get_state(psf_batch *B, int32_t basis, int32_t slot, double *w, int32_t n)
{
    int sg = 0;
    PSF_CHECK(slot_index(B, basis, slot, &sg));
    if (!w) return fail(PSF_ERR_INVALID, "null argument");
    const psf::SlotDev &s = B->slots[(size_t)sg];
    if (!s.active) return fail(PSF_ERR_STATE, "slot is empty");
    if (n != s.n_modes) return fail(PSF_ERR_INVALID, "n must equal the instance's n_modes");
    HostGroup &G = B->groups[(size_t)basis];
    PSF_CUDA(cudaSetDevice(B->device));
    PSF_CUDA(cudaMemcpyAsync(w, G.w + (size_t)slot * G.N, (size_t)n * 8, cudaMemcpyDeviceToHost, B->stream));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    return check_device_error(B);
}

int psf_batch_get_particles(psf_batch *B, int32_t basis, int32_t slot, float *xyzw, int64_t count)
{
    int sg = 0;
    PSF_CHECK(slot_index(B, basis, slot, &sg));
    const psf::SlotDev &s = B->slots[(size_t)sg];
    if (count != s.n_particles) return fail(PSF_ERR_INVALID, "count must equal the instance's particle count");
    if (count == 0) return PSF_OK;
    if (!xyzw) return fail(PSF_ERR_INVALID, "null argument");
    PSF_CUDA(cudaSetDevice(B->device));
    PSF_CHECK(psf::launch_unorder_particles(particle_view(B, basis, slot, count), B->order, B->stream));
    PSF_CUDA(cudaMemcpyAsync(xyzw, B->order.staging, (size_t)count * 16, cudaMemcpyDeviceToHost, B->stream));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    return check_device_error(B);
}

int psf_batch_get_velocity(psf_batch *B, int32_t basis, int32_t slot, float *u, int64_t n_faces)
{
    int sg = 0;
    PSF_CHECK(slot_index(B, basis, slot, &sg));
    HostGroup &G = B->groups[(size_t)basis];
    if (!u) return fail(PSF_ERR_INVALID, "null argument");
    if (n_faces != G.n_faces) return fail(PSF_ERR_INVALID, "n_faces must equal the grid's face count");
    PSF_CUDA(cudaSetDevice(B->device));
    // The slot's field lives in its per-voxel face pairs; every active face is
    // stored in both adjacent voxels, wall faces are zero.
    std::vector<float> pf;
    try {
        pf.resize((size_t)(6 * G.V));
    } catch (const std::bad_alloc &) {
        return fail(PSF_ERR_NOMEM, "host staging allocation failed");
    }
    PSF_CUDA(cudaMemcpyAsync(pf.data(), G.pairs + (size_t)slot * 3 * G.V, pf.size() * 4, cudaMemcpyDeviceToHost,
                             B->stream));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    std::fill(u, u + n_faces, 0.f);
    for (int64_t r = 0; r < G.F_act; ++r) {
        const int32_t face = G.faces_host[(size_t)r];
        const int32_t d = G.dst_host[(size_t)(2 * r)] >= 0 ? G.dst_host[(size_t)(2 * r)] : G.dst_host[(size_t)(2 * r + 1)];
        if (d >= 0) u[face] = pf[(size_t)d] * (float)G.sigma[(size_t)face];
    }
    return check_device_error(B);
}

int psf_batch_get_steps(psf_batch *B, int32_t basis, int32_t slot, int64_t *steps)
{
    int sg = 0;
    PSF_CHECK(slot_index(B, basis, slot, &sg));
    if (!steps) return fail(PSF_ERR_INVALID, "null argument");
    psf::SlotDev s{};
    PSF_CUDA(cudaSetDevice(B->device));
    PSF_CUDA(cudaMemcpyAsync(&s, B->d_slots + sg, sizeof(s), cudaMemcpyDeviceToHost, B->stream));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    *steps = (int64_t)s.step;
    return PSF_OK;
}

static int profile(psf_batch *B, double *kernel_ms, int32_t n, bool fused)
{
    const int nk = fused ? 2 : 4;
    if (n < nk) return fail(PSF_ERR_INVALID, "kernel_ms has fewer slots than launches per step");
    PSF_CUDA(cudaSetDevice(B->device));
    cudaEvent_t ev[5];
    for (int i = 0; i <= nk; ++i) PSF_CUDA(cudaEventCreate(&ev[i]));
    cudaStream_t st = B->stream;
    int rc = PSF_OK;
    cudaEventRecord(ev[0], st);
    if (fused) {
        rc = launch_tc_part(B, st, true);
        cudaEventRecord(ev[1], st);
    } else {
        rc = psf::launch_batch_step_tc(B->contract, B->bn_max, B->gemm_ctas, st);
        cudaEventRecord(ev[1], st);
        if (rc == PSF_OK) rc = psf::launch_batch_state(B->d_groups, B->d_slots, B->n_slots(), st);
        cudaEventRecord(ev[2], st);
        if (rc == PSF_OK) rc = psf::launch_batch_step_tc(B->recon, B->bn_max, B->gemm_ctas, st);
        cudaEventRecord(ev[3], st);
    }
    if (rc == PSF_OK)
        rc = psf::launch_batch_trace(B->d_groups, B->d_slots, B->d_prefix, B->n_slots(), B->trace_ctas, st);
    cudaEventRecord(ev[nk], st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == PSF_OK && e != cudaSuccess) rc = psf::cuda_fail(e, "profiled step");
    for (int i = 0; rc == PSF_OK && i < nk; ++i) {
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        if (e != cudaSuccess) rc = psf::cuda_fail(e, "cudaEventElapsedTime");
        kernel_ms[i] = ms;
    }
    for (int i = 0; i <= nk; ++i) cudaEventDestroy(ev[i]);
    if (rc == PSF_OK) rc = check_device_error(B);
    return rc;
}

int psf_batch_profile_step(psf_batch *B, double *kernel_ms, int32_t n)
{
    if (!B || !kernel_ms) return fail(PSF_ERR_INVALID, "null argument");
    return profile(B, kernel_ms, n, B->use_fused);
}

int psf_batch_profile_phases(psf_batch *B, double *kernel_ms, int32_t n)
{
    if (!B || !kernel_ms) return fail(PSF_ERR_INVALID, "null argument");
    PSF_CHECK(profile(B, kernel_ms, n, false));
    // A fused batch keeps the partials of its current state between steps.
    if (B->use_fused) {
        PSF_CHECK(psf::launch_batch_step_tc(B->contract, B->bn_max, B->gemm_ctas, B->stream));
        PSF_CUDA(cudaStreamSynchronize(B->stream));
    }
    return PSF_OK;
}

int psf_batch_device_status(psf_batch *B, int32_t *code)
{
    if (!B || !code) return fail(PSF_ERR_INVALID, "null argument");
    int c = 0;
    PSF_CUDA(cudaSetDevice(B->device));
    PSF_CUDA(cudaMemcpyAsync(&c, B->d_err, sizeof(int), cudaMemcpyDeviceToHost, B->stream));
    PSF_CUDA(cudaStreamSynchronize(B->stream));
    *code = c;
    return PSF_OK;
}

}  // extern "C"

namespace psf {

int batch_place_async(psf_batch *B, int32_t n, const int32_t *basis, const int32_t *slot,
                      const psf_instance_desc *const *inst, int32_t *status)
{
    if (!B || n < 0 || (n > 0 && (!basis || !slot || !inst || !status))) return fail(PSF_ERR_INVALID, "null argument");
    PSF_CUDA(cudaSetDevice(B->device));
    for (int32_t i = 0; i < n; ++i) status[i] = set_one(B, basis[i], slot[i], inst[i], B->kept_rows);
    return finish_placements(B, false);
}

int batch_prepare_reads(psf_batch *B)
{
    if (!B) return fail(PSF_ERR_INVALID, "null batch");
    PSF_CUDA(cudaSetDevice(B->device));
    if (!B->side) PSF_CUDA(cudaStreamCreateWithFlags(&B->side, cudaStreamNonBlocking));
    if (B->rd_cap < B->pmax_all) {
        float4 *parts = nullptr;
        int32_t *perm = nullptr;
        PSF_CUDA(cudaHostAlloc((void **)&parts, (size_t)B->pmax_all * 16, cudaHostAllocDefault));
        cudaError_t e = cudaHostAlloc((void **)&perm, (size_t)B->pmax_all * 4, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            cudaFreeHost(parts);
            return psf::cuda_fail(e, "cudaHostAlloc");
        }
        B->rd_parts = parts;
        B->rd_perm = perm;
        B->rd_cap = B->pmax_all;
    }
    return PSF_OK;
}

int batch_read_frozen(psf_batch *B, int32_t n, const int32_t *basis, const int32_t *slot, double *const *w,
                      float *const *xyzw)
{
    if (!B || n < 0 || (n > 0 && (!basis || !slot || !w || !xyzw))) return fail(PSF_ERR_INVALID, "null argument");
    if (!B->side || B->rd_cap < B->pmax_all) return fail(PSF_ERR_STATE, "frozen reads are not prepared");
    PSF_CUDA(cudaSetDevice(B->device));
    for (int32_t i = 0; i < n; ++i) {
        int sg = 0;
        PSF_CHECK(slot_index(B, basis[i], slot[i], &sg));
        const psf::SlotDev &s = B->slots[(size_t)sg];
        if (!s.active) return fail(PSF_ERR_STATE, "slot is empty");
        HostGroup &G = B->groups[(size_t)basis[i]];
        if (w[i])
            PSF_CUDA(cudaMemcpyAsync(w[i], G.w + (size_t)slot[i] * G.N, (size_t)s.n_modes * 8, cudaMemcpyDeviceToHost,
                                     B->side));
        const int64_t np = s.n_particles;
        if (xyzw[i] && np > 0) {
            PSF_CUDA(cudaMemcpyAsync(B->rd_parts, B->pool_parts + s.poff, (size_t)np * 16, cudaMemcpyDeviceToHost,
                                     B->side));
            PSF_CUDA(cudaMemcpyAsync(B->rd_perm, B->pool_perm + s.poff, (size_t)np * 4, cudaMemcpyDeviceToHost,
                                     B->side));
        }
        PSF_CUDA(cudaStreamSynchronize(B->side));
        if (xyzw[i] && np > 0) {
            float4 *out = reinterpret_cast<float4 *>(xyzw[i]);
            for (int64_t j = 0; j < np; ++j) {
                const int32_t d = B->rd_perm[j];
                if (d < 0 || d >= np) return fail(PSF_ERR_STATE, "particle order index out of range");
                out[d] = B->rd_parts[j];
            }
        }
    }
    return PSF_OK;
}

}  // namespace psf
