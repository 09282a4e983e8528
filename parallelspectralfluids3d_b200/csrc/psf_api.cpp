// C ABI of include/psf_b200.h: single-instance contexts.
//
// A context replaces the reference's PSFSolverGPU host object
// (Solver/SolverImpl/psfsolvergpu.cpp): it owns the device copies of the
// basis, the coefficient state, the face field and the particles, one CUDA
// stream, and a CUDA graph of one step.  Errors are returned as status codes
// (the reference prints and calls exit(), psfsolvergpu.cpp:39-104).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "psf_b200.h"
#include "psf_internal.h"

using psf::fail;

namespace {

inline int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

}  // namespace

namespace psf {

int64_t n_faces_of(const psf_grid &g)
{
    const int64_t nx = g.dims[0], ny = g.dims[1], nz = g.dims[2];
    return (nz + 1) * nx * ny + (ny + 1) * nx * nz + (nx + 1) * ny * nz;
}

// Per-face sign with which the reference tracer reads the face velocity
// (psfsolver.cpp:160-188): -s(v,4) / +s(v,5) for the x-faces at x / x+1 of
// voxel v, -s(v,2) / +s(v,3) for y, +s(v,0) / -s(v,1) for z, where s is
// DECMesh3D::getFaceSignum (DEC/decmesh3d.cpp:1848-1853).  Each face is read
// from up to two voxels; the readings must agree for the sign to be folded.
int fold_signs(const psf_grid &g, const uint32_t *bits, std::vector<int8_t> &sigma)
{
    const int64_t nx = g.dims[0], ny = g.dims[1], nz = g.dims[2];
    const int64_t yoff = (nz + 1) * nx * ny;
    const int64_t xoff = yoff + (ny + 1) * nx * nz;
    sigma.assign((size_t)n_faces_of(g), 0);
    auto sgn = [&](int64_t vid, int f) -> int {
        return ((bits[vid / 5] >> ((vid % 5) * 6 + f)) & 1u) ? 1 : -1;
    };
    auto put = [&](int64_t face, int s) -> bool {
        int8_t &d = sigma[(size_t)face];
        if (d != 0 && d != s) return false;
        d = (int8_t)s;
        return true;
    };
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const int64_t v = z * nx * ny + y * nx + x;
                bool ok = put(z * ny * (nx + 1) + y * (nx + 1) + x + xoff, -sgn(v, 4)) &&
                          put(z * ny * (nx + 1) + y * (nx + 1) + x + 1 + xoff, sgn(v, 5)) &&
                          put(z * (ny + 1) * nx + y * nx + x + yoff, -sgn(v, 2)) &&
                          put(z * (ny + 1) * nx + (y + 1) * nx + x + yoff, sgn(v, 3)) &&
                          put(z * nx * ny + y * nx + x, sgn(v, 0)) &&
                          put((z + 1) * nx * ny + y * nx + x, -sgn(v, 1));
                if (!ok) return fail(PSF_ERR_SIGNS, "face signs of two voxels disagree; cannot fold");
            }
    return PSF_OK;
}

void face_pair_slots(const psf_grid &g, const int32_t *faces, int64_t n_active, std::vector<int32_t> &dst)
{
    const int64_t nx = g.dims[0], ny = g.dims[1], nz = g.dims[2];
    const int64_t V = nx * ny * nz;
    const int64_t yoff = (nz + 1) * nx * ny;
    const int64_t xoff = yoff + (ny + 1) * nx * nz;
    dst.assign((size_t)(2 * n_active), -1);
    auto vox = [&](int64_t x, int64_t y, int64_t z) { return z * nx * ny + y * nx + x; };
    for (int64_t r = 0; r < n_active; ++r) {
        const int64_t f = faces[r];
        int64_t comp, x, y, z, lo_ok, hi_ok;
        if (f >= xoff) {  // x-face (x in 0..nx): pair .x of voxel x, pair .y of voxel x-1
            const int64_t t = f - xoff;
            z = t / (ny * (nx + 1));
            y = (t / (nx + 1)) % ny;
            x = t % (nx + 1);
            comp = 0;
            lo_ok = x < nx;
            hi_ok = x >= 1;
            dst[2 * r] = lo_ok ? (int32_t)(2 * (comp * V + vox(x, y, z))) : -1;
            dst[2 * r + 1] = hi_ok ? (int32_t)(2 * (comp * V + vox(x - 1, y, z)) + 1) : -1;
        } else if (f >= yoff) {  // y-face (y in 0..ny)
            const int64_t t = f - yoff;
            z = t / ((ny + 1) * nx);
            y = (t / nx) % (ny + 1);
            x = t % nx;
            comp = 1;
            lo_ok = y < ny;
            hi_ok = y >= 1;
            dst[2 * r] = lo_ok ? (int32_t)(2 * (comp * V + vox(x, y, z))) : -1;
            dst[2 * r + 1] = hi_ok ? (int32_t)(2 * (comp * V + vox(x, y - 1, z)) + 1) : -1;
        } else {  // z-face (z in 0..nz)
            z = f / (nx * ny);
            y = (f / nx) % ny;
            x = f % nx;
            comp = 2;
            lo_ok = z < nz;
            hi_ok = z >= 1;
            dst[2 * r] = lo_ok ? (int32_t)(2 * (comp * V + vox(x, y, z))) : -1;
            dst[2 * r + 1] = hi_ok ? (int32_t)(2 * (comp * V + vox(x, y, z - 1)) + 1) : -1;
        }
    }
}

psf::GridDev make_grid_dev(const psf_grid &g)
{
    GridDev d{};
    const int64_t nx = g.dims[0], ny = g.dims[1], nz = g.dims[2];
    d.nx = (int)nx;
    d.ny = (int)ny;
    d.nz = (int)nz;
    d.inv_h = (float)(1.0 / g.resolution);
    for (int q = 0; q < 3; ++q) {
        d.mn[q] = g.aabb_min[q];
        d.mx[q] = g.aabb_max[q];
        const float ext = g.aabb_max[q] - g.aabb_min[q];
        d.shift[q] = g.aabb_min[q] + ext;
    }
    d.centered = 1;
    for (int q = 0; q < 3; ++q)
        if (d.shift[q] != -d.mn[q]) d.centered = 0;
    d.yoff = (uint32_t)((nz + 1) * nx * ny);
    d.xoff = (uint32_t)((nz + 1) * nx * ny + (ny + 1) * nx * nz);
    return d;
}

}  // namespace psf

using psf::fold_signs;
using psf::n_faces_of;

// Software-pipelined step.  A context keeps three coefficient buffers (a ring)
// and two face-pair / velocity buffers.  Between steps, with the caller's
// state w^n in ring slot `vis` ("primed"): slot vis+1 holds w^{n+1}, slot
// vis+2 holds w^{n+2}, and face set `tq` holds the face pairs and velocity
// of w^{n+1}.  A step then runs, as three independent branches of one graph,
//   the tracer with face set tq                          (step n's particles)
//   the reconstruction of w^{n+2} into the other face set (step n+1's field)
//   the contraction of w^{n+2} into w^{n+3}, in slot vis  (step n+2's state)
// and the roles rotate.  Each kernel does one step's work of the reference's
// phase order, so results are bit-identical to running the phases one after
// the other.  Any change of state, forcing or parameters drops the lookahead
// ("unprimed").  The first step after such a change is a lean graph
// (contraction -> reconstruction -> tracer, nothing ahead), so a caller that
// resets the state before every step pays for no lookahead; a step taken
// while unprimed but with no change since the previous step is a bootstrap
// graph: the lean chain on the main branch and, beside it, the contractions
// and the reconstruction that prime the pipeline.  Every ring slot carries
// its step count; the tracer reads the count of a slot no kernel of the step
// writes.
struct psf_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t side[2] = {nullptr, nullptr};  // extra branches during graph capture
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr}, mid = nullptr, after_b = nullptr;
    cudaGraph_t graphs[3][6] = {};              // [lean, bootstrap, steady][vis * 2 + tq]
    cudaGraphExec_t execs[3][6] = {};
    double *wbuf[3] = {nullptr, nullptr, nullptr};
    unsigned long long *ctrbuf = nullptr;       // [3] completed steps of each slot's state
    float *ubuf[2] = {nullptr, nullptr};
    float2 *pbuf[2] = {nullptr, nullptr};
    int vis = 0, tq = 0;
    bool primed = false;
    bool changed = true;  // a setter ran since the last step
    int sets_since_sort = 0;  // psf_set_particles calls that reused the cell order
    bool have_state = false;
    // The contraction and reconstruction a lean step begins with, queued by
    // psf_set_particles on a side stream (they depend on the state only), for
    // the current ring position and inputs; a later setter drops them.
    bool eager = false;
    cudaEvent_t eager_fork = nullptr, eager_done = nullptr;
    cudaEvent_t h2d_done = nullptr;     // the caller's particles have crossed the bus
    double *wstage = nullptr;           // pinned copy of the last state set
    cudaEvent_t wstage_done = nullptr;  // ... and its upload
    psf_grid grid{};
    psf_params params{};
    std::vector<int8_t> sigma;
    psf::PlainDev d{};
    psf::OrderBufs order{};
    int32_t *perm = nullptr;
    std::vector<void *> allocs;

    ~psf_ctx()
    {
        drop_graph();
        for (void *p : allocs) cudaFree(p);
        for (cudaEvent_t e : {fork, join[0], join[1], mid, after_b, eager_fork, eager_done, h2d_done, wstage_done})
            if (e) cudaEventDestroy(e);
        if (wstage) cudaFreeHost(wstage);
        for (cudaStream_t s : side)
            if (s) cudaStreamDestroy(s);
        if (stream) cudaStreamDestroy(stream);
    }
    void drop_graph()
    {
        for (int k = 0; k < 3; ++k)
            for (int i = 0; i < 6; ++i) {
                if (execs[k][i]) cudaGraphExecDestroy(execs[k][i]);
                if (graphs[k][i]) cudaGraphDestroy(graphs[k][i]);
                execs[k][i] = nullptr;
                graphs[k][i] = nullptr;
            }
    }
    int slot(int k) const { return (vis + k) % 3; }
    static int slot_of(int v, int k) { return (v + k) % 3; }
    // Contraction of ring slot `from` into `to`.
    psf::PlainDev contraction(int from, int to) const
    {
        psf::PlainDev v = d;
        v.w = wbuf[from];
        v.w_next = wbuf[to];
        v.step_ctr = ctrbuf + from;
        v.step_ctr_next = ctrbuf + to;
        return v;
    }
    // Reconstruction of ring slot `from` into face set `fs`.
    psf::PlainDev reconstruction(int from, int fs) const
    {
        psf::PlainDev v = d;
        v.w = wbuf[from];
        v.u = ubuf[fs];
        v.pairs = pbuf[fs];
        return v;
    }
    // Tracer with face set `fs`, keyed by the step count of ring slot `from`.
    psf::PlainDev tracer(int from, int fs) const
    {
        psf::PlainDev v = d;
        v.trace_pairs = pbuf[fs];
        v.trace_ctr = ctrbuf + from;
        return v;
    }
    template <class T>
    int alloc(T **p, size_t count)
    {
        void *v = nullptr;
        cudaError_t e = cudaMalloc(&v, std::max<size_t>(1, count) * sizeof(T));
        if (e != cudaSuccess) return psf::cuda_fail(e, "cudaMalloc");
        allocs.push_back(v);
        *p = static_cast<T *>(v);
        return PSF_OK;
    }
    void release(void *p)
    {
        auto it = std::find(allocs.begin(), allocs.end(), p);
        if (it != allocs.end()) {
            cudaFree(p);
            allocs.erase(it);
        }
    }
};

#define PSF_CHECK(x)                  \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != PSF_OK) return rc_; \
    } while (0)
#define PSF_CUDA(x)                                      \
    do {                                                 \
        cudaError_t e_ = (x);                            \
        if (e_ != cudaSuccess) return psf::cuda_fail(e_, #x); \
    } while (0)

static int apply_params(psf_ctx *c, const psf_params &p)
{
    if (!(p.timestep > 0.0) || !std::isfinite(p.timestep))
        return fail(PSF_ERR_INVALID, "timestep must be positive and finite");
    if (p.integrator != PSF_RK1 && p.integrator != PSF_RK4)
        return fail(PSF_ERR_INVALID, "integrator must be PSF_RK1 or PSF_RK4");
    if (p.precision != PSF_PRECISION_FP32)
        return fail(PSF_ERR_UNSUPPORTED, "single-instance contexts store the basis in FP32");
    c->params = p;
    c->d.sp.dt = p.timestep;
    c->d.sp.visc_signed = (p.flags & PSF_FLAG_DECAY_NEG) ? -p.viscosity : p.viscosity;
    c->d.sp.flags = p.flags;
    c->d.tp.dt = (float)p.timestep;
    c->d.tp.lifetime = p.lifetime;
    c->d.tp.rk4 = p.integrator == PSF_RK4;
    c->d.tp.seed = p.seed;
    c->drop_graph();
    c->primed = false;
    c->changed = true;
    c->eager = false;
    return PSF_OK;
}

// Synchronise the context's stream.
static int sync_stream(psf_ctx *c)
{
    PSF_CUDA(cudaStreamSynchronize(c->stream));
    return PSF_OK;
}

enum StepKind { STEP_LEAN = 0, STEP_BOOT = 1, STEP_STEADY = 2 };

// Capture one step of the given kind, for ring position (v, q), into a graph.
static int capture_step(psf_ctx *c, int kind, int v, int q, cudaGraph_t *out)
{
    const int v0 = psf_ctx::slot_of(v, 0), v1 = psf_ctx::slot_of(v, 1), v2 = psf_ctx::slot_of(v, 2);
    cudaStream_t m = c->stream, s0 = c->side[0], s1 = c->side[1];
    int rc = PSF_OK;
    auto ok = [&](cudaError_t e, const char *what) {
        if (rc == PSF_OK && e != cudaSuccess) rc = psf::cuda_fail(e, what);
        return rc == PSF_OK;
    };
    if (!ok(cudaStreamBeginCapture(m, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture")) return rc;
    bool forked = false;
    if (kind == STEP_STEADY) {
        // step n's particles, step n+1's field, step n+2's state: three independent branches.
        forked = ok(cudaEventRecord(c->fork, m), "fork") && ok(cudaStreamWaitEvent(s0, c->fork, 0), "fork") &&
                 ok(cudaStreamWaitEvent(s1, c->fork, 0), "fork");
        if (forked) {
            rc = psf::launch_reconstruct(c->reconstruction(v2, 1 - q), s0, /*after_kernel=*/false);
            if (rc == PSF_OK) rc = psf::launch_contract_state(c->contraction(v2, v0), s1);
            if (rc == PSF_OK) rc = psf::launch_trace(c->tracer(v1, q), m, /*after_kernel=*/false);
        }
    } else {
        // main: w^{n+1}, its field, step n's particles.
        rc = psf::launch_contract_state(c->contraction(v0, v1), m);
        if (rc == PSF_OK && kind == STEP_BOOT) {
            // beside it: w^{n+2}, its field, w^{n+3}.
            forked = ok(cudaEventRecord(c->mid, m), "fork") && ok(cudaStreamWaitEvent(s0, c->mid, 0), "fork");
            if (forked) {
                rc = psf::launch_contract_state(c->contraction(v1, v2), s0);
                if (rc == PSF_OK && ok(cudaEventRecord(c->after_b, s0), "fork") &&
                    ok(cudaStreamWaitEvent(s1, c->after_b, 0), "fork"))
                    rc = psf::launch_reconstruct(c->reconstruction(v2, 1 - q), s1, /*after_kernel=*/false);
                if (rc == PSF_OK) rc = psf::launch_contract_state(c->contraction(v2, v0), s0);
            }
        }
        if (rc == PSF_OK) rc = psf::launch_reconstruct(c->reconstruction(v1, q), m, /*after_kernel=*/true);
        if (rc == PSF_OK) rc = psf::launch_trace(c->tracer(v1, q), m, /*after_kernel=*/true);
    }
    if (rc == PSF_OK && forked) {
        ok(cudaEventRecord(c->join[0], s0), "join") && ok(cudaStreamWaitEvent(m, c->join[0], 0), "join") &&
            ok(cudaEventRecord(c->join[1], s1), "join") && ok(cudaStreamWaitEvent(m, c->join[1], 0), "join");
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(m, &g);
    if (rc != PSF_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return psf::cuda_fail(e, "cudaStreamEndCapture");
    *out = g;
    return PSF_OK;
}

// Launch one step and rotate the ring.  The six ring positions of a step
// kind are captured together, the first time that kind is needed.
static int launch_step(psf_ctx *c)
{
    const int kind = c->primed ? STEP_STEADY : (c->changed ? STEP_LEAN : STEP_BOOT);
    const int idx = c->vis * 2 + c->tq;
    if (kind == STEP_LEAN && c->eager) {
        // The lean step's contraction and reconstruction are already queued
        // (psf_set_particles); its tracer remains.
        PSF_CHECK(psf::launch_trace(c->tracer(c->slot(1), c->tq), c->stream, /*after_kernel=*/false));
        c->vis = c->slot(1);
        c->tq = 1 - c->tq;
        c->primed = false;
        c->changed = false;
        c->eager = false;
        return PSF_OK;
    }
    if (!c->execs[kind][idx]) {
        for (int v = 0; v < 3; ++v)
            for (int q = 0; q < 2; ++q) {
                const int i = v * 2 + q;
                if (c->execs[kind][i]) continue;
                cudaGraph_t g = nullptr;
                PSF_CHECK(capture_step(c, kind, v, q, &g));
                c->graphs[kind][i] = g;
                PSF_CUDA(cudaGraphInstantiate(&c->execs[kind][i], g, 0));
            }
    }
    PSF_CUDA(cudaGraphLaunch(c->execs[kind][idx], c->stream));
    c->vis = c->slot(1);
    c->tq = 1 - c->tq;
    c->primed = kind != STEP_LEAN;
    c->changed = false;
    return PSF_OK;
}

int psf::context_particles(psf_ctx *c, ContextParticles *out)
{
    if (!c || !out) return fail(PSF_ERR_INVALID, "null argument");
    out->device = c->device;
    out->stream = c->stream;
    out->parts = c->d.parts;
    out->n = c->d.P;
    for (int a = 0; a < 3; ++a) {
        out->mn[a] = c->grid.aabb_min[a];
        out->mx[a] = c->grid.aabb_max[a];
    }
    return PSF_OK;
}

extern "C" {

int psf_abi_version(void) { return PSF_ABI_VERSION; }

const char *psf_last_error(void) { return psf::g_last_error.c_str(); }

int psf_device_count(int *count)
{
    if (!count) return fail(PSF_ERR_INVALID, "count is null");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return PSF_OK;
}

int psf_create(const psf_basis_desc *b, const psf_params *params, int device, psf_ctx **out)
{
    if (!b || !params || !out) return fail(PSF_ERR_INVALID, "null argument");
    *out = nullptr;
    const psf_grid &g = b->grid;
    if (g.dims[0] == 0 || g.dims[1] == 0 || g.dims[2] == 0 || !(g.resolution > 0.0))
        return fail(PSF_ERR_INVALID, "grid dims and resolution must be positive");
    if (g.dims[0] > 1023 || g.dims[1] > 1023 || g.dims[2] > 1023)
        return fail(PSF_ERR_UNSUPPORTED, "grid dims above 1023 voxels per axis");
    if (b->n_modes < 1 || b->n_modes > psf::PSF_MAX_MODES)
        return fail(PSF_ERR_UNSUPPORTED, "n_modes must be in [1, 1024]");
    if (b->n_active < 1) return fail(PSF_ERR_INVALID, "n_active must be positive");
    if (!b->active_faces || !b->phi || !b->advection || !b->eigenvalues || !b->sign_bits)
        return fail(PSF_ERR_INVALID, "basis arrays must not be null");
    const int64_t F = n_faces_of(g);
    const int64_t V = (int64_t)g.dims[0] * g.dims[1] * g.dims[2];
    if (F >= (int64_t)UINT32_MAX || 6 * V >= (int64_t)INT32_MAX)
        return fail(PSF_ERR_UNSUPPORTED, "grid has too many faces");
    for (int64_t r = 0; r < b->n_active; ++r)
        if (b->active_faces[r] < 0 || b->active_faces[r] >= F)
            return fail(PSF_ERR_INVALID, "active face id out of range");

    psf_ctx *c = nullptr;
    try {
        c = new psf_ctx();
    } catch (const std::bad_alloc &) {
        return fail(PSF_ERR_NOMEM, "host allocation failed");
    }
    auto bail = [&](int rc) {
        delete c;
        return rc;
    };
    int rc = PSF_OK;
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(psf::cuda_fail(e, "cudaSetDevice"));
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    for (cudaStream_t *s : {&c->side[0], &c->side[1]})
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
    for (cudaEvent_t *ev : {&c->fork, &c->join[0], &c->join[1], &c->mid, &c->after_b, &c->eager_fork,
                            &c->eager_done, &c->h2d_done, &c->wstage_done})
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return bail(psf::cuda_fail(e, "cudaStreamCreate"));
    c->grid = g;
    if ((rc = fold_signs(g, b->sign_bits, c->sigma)) != PSF_OK) return bail(rc);

    psf::PlainDev &d = c->d;
    const int N = b->n_modes;
    d.N = N;
    d.Np = (int)round_up(N, 4);
    d.S = std::max(1, std::min(N, (2 * c->num_sms + N - 1) / N));
    d.n_active = b->n_active;
    d.ldp = round_up(b->n_active, 64);  // whole 64-face tiles
    d.n_faces = F;
    d.P = 0;

    try {
        // C as FP32 [k][a][j] with j padded to Np.
        std::vector<float> hC((size_t)N * N * d.Np, 0.f);
        for (int64_t ka = 0; ka < (int64_t)N * N; ++ka)
            for (int j = 0; j < N; ++j) hC[(size_t)ka * d.Np + j] = (float)b->advection[(size_t)ka * N + j];
        // Phi as tiles of 64 faces, each tile mode-major ([tile][i][face in tile]),
        // so one tile's modes are contiguous in memory; the tracer's face signs
        // are folded in.
        std::vector<float> hP((size_t)N * d.ldp, 0.f);
        for (int64_t r = 0; r < b->n_active; ++r) {
            const float s = (float)c->sigma[(size_t)b->active_faces[r]];
            const size_t base = (size_t)(r / 64) * N * 64 + (size_t)(r % 64);
            for (int i = 0; i < N; ++i) hP[base + (size_t)i * 64] = s * (float)b->phi[(size_t)r * N + i];
        }
        float *C = nullptr, *phiT = nullptr;
        int32_t *faces = nullptr;
        double *lam = nullptr, *force = nullptr;
        if ((rc = c->alloc(&C, hC.size())) || (rc = c->alloc(&phiT, hP.size())) ||
            (rc = c->alloc(&faces, (size_t)b->n_active)) || (rc = c->alloc(&c->wbuf[0], 3 * (size_t)N)) ||
            (rc = c->alloc(&d.dwpart, (size_t)N * d.S)) || (rc = c->alloc(&lam, (size_t)N)) ||
            (rc = c->alloc(&force, (size_t)N)) || (rc = c->alloc(&d.ticket, 1)) ||
            (rc = c->alloc(&c->ctrbuf, 3)) || (rc = c->alloc(&c->ubuf[0], 2 * (size_t)F)))
            return bail(rc);
        c->wbuf[1] = c->wbuf[0] + N;
        c->wbuf[2] = c->wbuf[0] + 2 * N;
        c->ubuf[1] = c->ubuf[0] + F;
        e = cudaHostAlloc((void **)&c->wstage, (size_t)N * 8, cudaHostAllocDefault);
        if (e != cudaSuccess) return bail(psf::cuda_fail(e, "cudaHostAlloc"));
        // Per-voxel face pairs read by the tracer, and where each active face goes.
        std::vector<int32_t> hdst;
        psf::face_pair_slots(g, b->active_faces, b->n_active, hdst);
        int32_t *pdst = nullptr;
        if ((rc = c->alloc(&c->pbuf[0], (size_t)(6 * V))) || (rc = c->alloc(&pdst, hdst.size()))) return bail(rc);
        c->pbuf[1] = c->pbuf[0] + 3 * V;
        d.pair_dst = pdst;
        if ((e = cudaMemsetAsync(c->pbuf[0], 0, (size_t)(6 * V) * sizeof(float2), c->stream)) ||
            (e = cudaMemcpyAsync(pdst, hdst.data(), hdst.size() * 4, cudaMemcpyHostToDevice, c->stream)) ||
            (e = cudaStreamSynchronize(c->stream)))
            return bail(psf::cuda_fail(e, "face pair upload"));
        d.C = C;
        d.phiT = phiT;
        d.faces = faces;
        d.lam = lam;
        d.force = force;
        cudaStream_t st = c->stream;
        if ((e = cudaMemcpyAsync(C, hC.data(), hC.size() * 4, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(phiT, hP.data(), hP.size() * 4, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(faces, b->active_faces, (size_t)b->n_active * 4, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(lam, b->eigenvalues, (size_t)N * 8, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemsetAsync(force, 0, (size_t)N * 8, st)) ||
            (e = cudaMemsetAsync(c->wbuf[0], 0, 3 * (size_t)N * 8, st)) ||
            (e = cudaMemsetAsync(d.ticket, 0, 4, st)) || (e = cudaMemsetAsync(c->ctrbuf, 0, 24, st)) ||
            (e = cudaMemsetAsync(c->ubuf[0], 0, 2 * (size_t)F * 4, st)) || (e = cudaStreamSynchronize(st)))
            return bail(psf::cuda_fail(e, "basis upload"));
    } catch (const std::bad_alloc &) {
        return bail(fail(PSF_ERR_NOMEM, "host staging allocation failed"));
    }

    d.grid = psf::make_grid_dev(g);
    d.trace_blocks = c->num_sms * psf::trace_blocks_per_sm();
    if ((rc = apply_params(c, *params)) != PSF_OK) return bail(rc);
    *out = c;
    return PSF_OK;
}

int psf_destroy(psf_ctx *c)
{
    if (!c) return PSF_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    delete c;
    return PSF_OK;
}

int psf_set_params(psf_ctx *c, const psf_params *p)
{
    if (!c || !p) return fail(PSF_ERR_INVALID, "null argument");
    if (p->precision != c->params.precision)
        return fail(PSF_ERR_INVALID, "precision is fixed when the context is created");
    return apply_params(c, *p);
}

int psf_set_state(psf_ctx *c, const double *w, int32_t n)
{
    if (!c || !w) return fail(PSF_ERR_INVALID, "null argument");
    if (n != c->d.N) return fail(PSF_ERR_INVALID, "state length must equal n_modes");
    PSF_CUDA(cudaSetDevice(c->device));
    // Through a pinned copy: the caller's buffer is free on return, and the
    // call does not wait for the stream.
    PSF_CUDA(cudaEventSynchronize(c->wstage_done));
    std::memcpy(c->wstage, w, (size_t)n * 8);
    PSF_CUDA(cudaMemcpyAsync(c->wbuf[c->vis], c->wstage, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
    PSF_CUDA(cudaEventRecord(c->wstage_done, c->stream));
    c->primed = false;
    c->changed = true;
    c->eager = false;
    c->have_state = true;
    return PSF_OK;
}

int psf_get_state(psf_ctx *c, double *w, int32_t n)
{
    if (!c || !w) return fail(PSF_ERR_INVALID, "null argument");
    if (n != c->d.N) return fail(PSF_ERR_INVALID, "state length must equal n_modes");
    PSF_CUDA(cudaSetDevice(c->device));
    PSF_CUDA(cudaMemcpyAsync(w, c->wbuf[c->vis], (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
    PSF_CHECK(sync_stream(c));
    return PSF_OK;
}

int psf_set_forcing(psf_ctx *c, const double *f, int32_t n)
{
    if (!c || !f) return fail(PSF_ERR_INVALID, "null argument");
    if (n != c->d.N) return fail(PSF_ERR_INVALID, "forcing length must equal n_modes");
    PSF_CUDA(cudaSetDevice(c->device));
    PSF_CUDA(cudaMemcpyAsync(const_cast<double *>(c->d.force), f, (size_t)n * 8, cudaMemcpyHostToDevice,
                             c->stream));
    PSF_CUDA(cudaStreamSynchronize(c->stream));
    c->primed = false;
    c->changed = true;
    c->eager = false;
    return PSF_OK;
}

int psf_set_particles(psf_ctx *c, const float *xyzw, int64_t count)
{
    if (!c || (count > 0 && !xyzw)) return fail(PSF_ERR_INVALID, "null argument");
    if (count < 0 || count > INT32_MAX) return fail(PSF_ERR_INVALID, "bad particle count");
    PSF_CUDA(cudaSetDevice(c->device));
    const bool resized = count != c->d.P;
    if (resized) {
        PSF_CUDA(cudaStreamSynchronize(c->stream));
        c->drop_graph();
        psf::OrderBufs &o = c->order;
        for (void *p : {(void *)c->d.parts, (void *)c->perm, (void *)o.staging, (void *)o.keys_in,
                        (void *)o.keys_out, (void *)o.idx_in, o.temp})
            if (p) c->release(p);
        c->d.parts = nullptr;
        c->perm = nullptr;
        c->d.perm = nullptr;
        o = psf::OrderBufs{};
        c->d.P = 0;
        if (count > 0) {
            size_t tmp = 0;
            PSF_CHECK(psf::sort_particles_temp_bytes(count, &tmp));
            unsigned char *temp = nullptr;
            PSF_CHECK(c->alloc(&c->d.parts, (size_t)count));
            PSF_CHECK(c->alloc(&c->perm, (size_t)count));
            PSF_CHECK(c->alloc(&o.staging, (size_t)count));
            PSF_CHECK(c->alloc(&o.keys_in, (size_t)count));
            PSF_CHECK(c->alloc(&o.keys_out, (size_t)count));
            PSF_CHECK(c->alloc(&o.idx_in, (size_t)count));
            PSF_CHECK(c->alloc(&temp, tmp));
            o.temp = temp;
            o.temp_bytes = tmp;
            c->d.perm = c->perm;
        }
        c->d.P = count;
    }
    if (count > 0) {
        // The same particles set again (an end-to-end loop) are still close to
        // the cell order of the last sort: reuse it, and sort afresh on a new
        // count and on every RESORT_EVERY-th call.  Results do not depend on the
        // storage order (respawns are keyed by the caller's index).
        constexpr int RESORT_EVERY = 8;
        const bool resort = resized || c->sets_since_sort + 1 >= RESORT_EVERY;
        // A lean step comes next (the state changed): its contraction and
        // reconstruction depend on the state only, so they are queued now on
        // a side stream and run while the particles cross the bus.
        const bool eager_now = c->have_state && c->changed && !c->primed && !c->eager;
        if (eager_now) {
            PSF_CUDA(cudaEventRecord(c->eager_fork, c->stream));
            PSF_CUDA(cudaStreamWaitEvent(c->side[0], c->eager_fork, 0));
            PSF_CHECK(psf::launch_contract_state(c->contraction(c->slot(0), c->slot(1)), c->side[0]));
            PSF_CHECK(psf::launch_reconstruct(c->reconstruction(c->slot(1), c->tq), c->side[0],
                                              /*after_kernel=*/true));
            PSF_CUDA(cudaEventRecord(c->eager_done, c->side[0]));
        }
        PSF_CUDA(cudaMemcpyAsync(c->order.staging, xyzw, (size_t)count * 16, cudaMemcpyHostToDevice, c->stream));
        PSF_CUDA(cudaEventRecord(c->h2d_done, c->stream));
        PSF_CHECK(psf::launch_order_particles(c->d, c->order, c->stream, resort));
        c->sets_since_sort = resort ? 0 : c->sets_since_sort + 1;
        if (eager_now) {
            PSF_CUDA(cudaStreamWaitEvent(c->stream, c->eager_done, 0));
            c->eager = true;
        }
        // Return once the caller's buffer has been read; the ordering (and the
        // queued lookahead) finish on the stream.
        PSF_CUDA(cudaEventSynchronize(c->h2d_done));
    }
    return PSF_OK;
}

int psf_get_particles(psf_ctx *c, float *xyzw, int64_t count)
{
    if (!c || (count > 0 && !xyzw)) return fail(PSF_ERR_INVALID, "null argument");
    if (count != c->d.P) return fail(PSF_ERR_INVALID, "count must equal the number of particles");
    if (count == 0) return PSF_OK;
    PSF_CUDA(cudaSetDevice(c->device));
    PSF_CHECK(psf::launch_unorder_particles(c->d, c->order, c->stream));
    PSF_CUDA(cudaMemcpyAsync(xyzw, c->order.staging, (size_t)count * 16, cudaMemcpyDeviceToHost, c->stream));
    PSF_CHECK(sync_stream(c));
    return PSF_OK;
}

int psf_get_velocity(psf_ctx *c, float *u, int64_t n_faces)
{
    if (!c || !u) return fail(PSF_ERR_INVALID, "null argument");
    if (n_faces != c->d.n_faces) return fail(PSF_ERR_INVALID, "n_faces must equal the grid's face count");
    PSF_CUDA(cudaSetDevice(c->device));
    PSF_CUDA(cudaMemcpyAsync(u, c->ubuf[1 - c->tq], (size_t)n_faces * 4, cudaMemcpyDeviceToHost, c->stream));
    PSF_CHECK(sync_stream(c));
    for (int64_t f = 0; f < n_faces; ++f) u[f] *= (float)c->sigma[(size_t)f];
    return PSF_OK;
}

int psf_step(psf_ctx *c, int32_t nsteps)
{
    if (!c) return fail(PSF_ERR_INVALID, "null context");
    if (nsteps < 0) return fail(PSF_ERR_INVALID, "nsteps must be >= 0");
    if (!c->have_state) return fail(PSF_ERR_STATE, "psf_set_state must be called before stepping");
    PSF_CUDA(cudaSetDevice(c->device));
    for (int32_t i = 0; i < nsteps; ++i) PSF_CHECK(launch_step(c));
    return PSF_OK;
}

int psf_sync(psf_ctx *c)
{
    if (!c) return fail(PSF_ERR_INVALID, "null context");
    PSF_CUDA(cudaSetDevice(c->device));
    return sync_stream(c);
}

int psf_get_stream(psf_ctx *c, void **stream)
{
    if (!c || !stream) return fail(PSF_ERR_INVALID, "null argument");
    *stream = (void *)c->stream;
    return PSF_OK;
}

int psf_kernels_per_step(psf_ctx *c, int32_t *count)
{
    if (!c || !count) return fail(PSF_ERR_INVALID, "null argument");
    *count = c->d.P > 0 ? 3 : 2;
    return PSF_OK;
}

int psf_profile_step(psf_ctx *c, double *kernel_ms, int32_t n)
{
    if (!c || !kernel_ms) return fail(PSF_ERR_INVALID, "null argument");
    if (!c->have_state) return fail(PSF_ERR_STATE, "psf_set_state must be called before stepping");
    const int nk = c->d.P > 0 ? 3 : 2;
    if (n < nk) return fail(PSF_ERR_INVALID, "kernel_ms has fewer slots than kernels per step");
    PSF_CUDA(cudaSetDevice(c->device));
    cudaEvent_t ev[4];
    for (int i = 0; i <= nk; ++i) PSF_CUDA(cudaEventCreate(&ev[i]));
    int rc = PSF_OK;
    cudaStream_t st = c->stream;
    // The kernels of one (steady) step, one after the other: the contraction
    // of w^{n+3}, the reconstruction of w^{n+2}, the tracer of step n.  An
    // unprimed pipeline is primed first, untimed.
    if (!c->primed) {
        rc = psf::launch_contract_state(c->contraction(c->slot(0), c->slot(1)), st);
        if (rc == PSF_OK) rc = psf::launch_contract_state(c->contraction(c->slot(1), c->slot(2)), st);
        if (rc == PSF_OK) rc = psf::launch_reconstruct(c->reconstruction(c->slot(1), c->tq), st, false);
        if (rc == PSF_OK) c->primed = true;
    }
    cudaEventRecord(ev[0], st);
    if (rc == PSF_OK) rc = psf::launch_contract_state(c->contraction(c->slot(2), c->slot(0)), st);
    cudaEventRecord(ev[1], st);
    if (rc == PSF_OK) rc = psf::launch_reconstruct(c->reconstruction(c->slot(2), 1 - c->tq), st, false);
    cudaEventRecord(ev[2], st);
    if (rc == PSF_OK && nk == 3) {
        rc = psf::launch_trace(c->tracer(c->slot(1), c->tq), st, false);
        cudaEventRecord(ev[3], st);
    }
    if (rc == PSF_OK) {
        c->vis = c->slot(1);
        c->tq = 1 - c->tq;
        c->changed = false;
        c->eager = false;
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == PSF_OK && e != cudaSuccess) rc = psf::cuda_fail(e, "profiled step");
    for (int i = 0; rc == PSF_OK && i < nk; ++i) {
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
        if (e != cudaSuccess) rc = psf::cuda_fail(e, "cudaEventElapsedTime");
        kernel_ms[i] = ms;
    }
    for (int i = 0; i <= nk; ++i) cudaEventDestroy(ev[i]);
    return rc;
}

}  // extern "C"
