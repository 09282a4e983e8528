/*
 * Test infrastructure (oracle) -- FP64 CPU restatement of the reference's
 * per-step spectral-fluid path.  Only the tests, the smoke check and the CPU
 * baseline leg of the benchmark load this library; it is the checker, never
 * the product path.
 *
 * Follows Solver/SolverImpl/psfsolver.cpp (PSFSolver::integrate):
 *   psfo_coeff_step   :34-59  e1 = w.w; dw_k = (w^T C_k) w; w += dt dw;
 *                              e2 = w.w; w *= sqrt(e1/e2); w_k *= exp(nu lam_k dt);
 *                              w += dt g
 *   psfo_reconstruct  :60     u = float(Phi w)
 *   psfo_trace        :75-224 particle loop: truncating voxel offsets,
 *                              clamp, DECMesh3D index functions, sign-bit
 *                              lookups, glm::mix trilinear (weights not
 *                              clamped), p = clamp(p + dt v, aabb), life -= 1,
 *                              respawn when life <= 0.
 * Index and sign functions: DEC/decmesh3d.cpp:12-30, 1848-1853.
 *
 * Extensions of the reference (flags): RK4 stages (each stage position is
 * clamped to the box like the final one), the GPU kernel's decay sign
 * exp(-nu lam dt) (Resources/Simulation/simulation.cl:211), and a
 * deterministic counter-based respawn generator in place of rand().
 *
 * Parity unpinned: the reference ships no tests, golden vectors or fixtures
 * for this path and cannot be compiled here (Eigen3, glm, OpenCL and Qt are
 * absent), so this restatement is checked against independent NumPy
 * restatements and known answers only.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PSFO_FLAG_RENORM 1u
#define PSFO_FLAG_DECAY_NEG 2u
#define PSFO_FLAG_FORCING 4u

typedef struct psfo_grid {
    uint32_t dims[3];
    double h;
    float aabb_min[3];
    float aabb_max[3];
} psfo_grid;

int psfo_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void psfo_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ coeffs */
void psfo_contract(int32_t N, const double *C, const double *w, double *dw)
{
    /* dw_k = (w^T C_k) w, psfsolver.cpp:40-44 (Eigen evaluates w^T C_k first). */
#pragma omp parallel for schedule(static)
    for (int32_t k = 0; k < N; ++k) {
        const double *Ck = C + (size_t)k * N * N;
        double acc = 0.0;
        for (int32_t j = 0; j < N; ++j) {
            double t = 0.0;
            for (int32_t a = 0; a < N; ++a) t += w[a] * Ck[(size_t)a * N + j];
            acc += t * w[j];
        }
        dw[k] = acc;
    }
}

void psfo_coeff_step(int32_t N, const double *C, const double *lam, const double *force,
                     double dt, double visc, uint32_t flags, double *w, double *dw)
{
    double e1 = 0.0, e2 = 0.0;
    for (int32_t i = 0; i < N; ++i) e1 += w[i] * w[i];
    psfo_contract(N, C, w, dw);
    for (int32_t i = 0; i < N; ++i) w[i] += dt * dw[i];
    for (int32_t i = 0; i < N; ++i) e2 += w[i] * w[i];
    if (flags & PSFO_FLAG_RENORM) {
        double s = sqrt(e1 / e2);
        for (int32_t i = 0; i < N; ++i) w[i] *= s;
    }
    double sgn = (flags & PSFO_FLAG_DECAY_NEG) ? -1.0 : 1.0;
    for (int32_t i = 0; i < N; ++i) w[i] *= exp(sgn * visc * lam[i] * dt);
    if ((flags & PSFO_FLAG_FORCING) && force)
        for (int32_t i = 0; i < N; ++i) w[i] += dt * force[i];
}

/* u = float(Phi w) on the active faces, 0 elsewhere (psfsolver.cpp:60). */
void psfo_reconstruct(int64_t n_active, int32_t N, const double *phi, const int32_t *faces,
                      int64_t n_faces, const double *w, float *u)
{
    memset(u, 0, sizeof(float) * (size_t)n_faces);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n_active; ++r) {
        const double *row = phi + (size_t)r * N;
        double acc = 0.0;
        for (int32_t i = 0; i < N; ++i) acc += row[i] * w[i];
        u[faces[r]] = (float)acc;
    }
}

/* ------------------------------------------------------------------ tracer */
static inline uint32_t vox_idx(const uint32_t *d, uint32_t x, uint32_t y, uint32_t z)
{
    return z * (d[0] * d[1]) + y * d[0] + x;
}
static inline uint32_t zface_idx(const uint32_t *d, uint32_t x, uint32_t y, uint32_t z)
{
    return z * (d[0] * d[1]) + y * d[0] + x;
}
static inline uint32_t yface_idx(const uint32_t *d, uint32_t x, uint32_t y, uint32_t z)
{
    return z * ((d[1] + 1) * d[0]) + y * d[0] + x + (d[2] + 1) * (d[0] * d[1]);
}
static inline uint32_t xface_idx(const uint32_t *d, uint32_t x, uint32_t y, uint32_t z)
{
    return z * (d[1] * (d[0] + 1)) + y * (d[0] + 1) + x + (d[2] + 1) * (d[0] * d[1]) +
           (d[1] + 1) * (d[0] * d[2]);
}
static inline int face_signum(const uint32_t *bits, uint32_t vid, uint32_t fidx)
{
    return (bits[vid / 5] >> ((vid % 5) * 6 + fidx)) & 1u ? 1 : -1;
}
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline double mixd(double x, double y, double a) { return x * (1.0 - a) + y * a; }
static inline double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Velocity at p, literal restatement of psfsolver.cpp:80-212. */
static void velocity_at(const psfo_grid *g, const float *u, const uint32_t *bits, const double p[3],
                        double v[3])
{
    const uint32_t *d = g->dims;
    const double h = g->h;
    double shift[3];
    for (int c = 0; c < 3; ++c) {
        /* min + extent, evaluated in float as glm::vec3 arithmetic does. */
        float ext = g->aabb_max[c] - g->aabb_min[c];
        shift[c] = (double)(g->aabb_min[c] + ext);
    }
    int xO = (int)((shift[0] + p[0]) / h);
    int yO = (int)((shift[1] + p[1]) / h);
    int zO = (int)((shift[2] + p[2]) / h);
    int zM = (int)((shift[2] + p[2] - h / 2) / h);
    int zP = (int)((shift[2] + p[2] + h / 2) / h);
    int yM = (int)((shift[1] + p[1] - h / 2) / h);
    int yP = (int)((shift[1] + p[1] + h / 2) / h);
    int xM = (int)((shift[0] + p[0] - h / 2) / h);
    int xP = (int)((shift[0] + p[0] + h / 2) / h);
    xO = clampi(xO, 0, (int)d[0] - 1);
    yO = clampi(yO, 0, (int)d[1] - 1);
    zO = clampi(zO, 0, (int)d[2] - 1);
    xM = clampi(xM, 0, (int)d[0] - 1);
    xP = clampi(xP, 0, (int)d[0] - 1);
    yM = clampi(yM, 0, (int)d[1] - 1);
    yP = clampi(yP, 0, (int)d[1] - 1);
    zM = clampi(zM, 0, (int)d[2] - 1);
    zP = clampi(zP, 0, (int)d[2] - 1);

    uint32_t v1x = vox_idx(d, xO, yM, zM), v2x = vox_idx(d, xO, yP, zM);
    uint32_t v3x = vox_idx(d, xO, yM, zP), v4x = vox_idx(d, xO, yP, zP);
    uint32_t v1y = vox_idx(d, xM, yO, zM), v2y = vox_idx(d, xP, yO, zM);
    uint32_t v3y = vox_idx(d, xM, yO, zP), v4y = vox_idx(d, xP, yO, zP);
    uint32_t v1z = vox_idx(d, xM, yM, zO), v2z = vox_idx(d, xP, yM, zO);
    uint32_t v3z = vox_idx(d, xM, yP, zO), v4z = vox_idx(d, xP, yP, zO);

    double mn[3] = {g->aabb_min[0], g->aabb_min[1], g->aabb_min[2]};
    double cfx[3] = {mn[0] + h * xO, mn[1] + h * yM + 0.5 * h, mn[2] + h * zM + 0.5 * h};
    double cfy[3] = {mn[0] + h * xM + 0.5 * h, mn[1] + h * yO, mn[2] + h * zM + 0.5 * h};
    double cfz[3] = {mn[0] + h * xM + 0.5 * h, mn[1] + h * yM + 0.5 * h, mn[2] + h * zO};

    double X1 = -face_signum(bits, v1x, 4) * (double)u[xface_idx(d, xO, yM, zM)];
    double X3 = face_signum(bits, v1x, 5) * (double)u[xface_idx(d, xO + 1, yM, zM)];
    double X2 = -face_signum(bits, v2x, 4) * (double)u[xface_idx(d, xO, yP, zM)];
    double X4 = face_signum(bits, v2x, 5) * (double)u[xface_idx(d, xO + 1, yP, zM)];
    double X5 = -face_signum(bits, v3x, 4) * (double)u[xface_idx(d, xO, yM, zP)];
    double X7 = face_signum(bits, v3x, 5) * (double)u[xface_idx(d, xO + 1, yM, zP)];
    double X6 = -face_signum(bits, v4x, 4) * (double)u[xface_idx(d, xO, yP, zP)];
    double X8 = face_signum(bits, v4x, 5) * (double)u[xface_idx(d, xO + 1, yP, zP)];

    double Y1 = -face_signum(bits, v1y, 2) * (double)u[yface_idx(d, xM, yO, zM)];
    double Y2 = face_signum(bits, v1y, 3) * (double)u[yface_idx(d, xM, yO + 1, zM)];
    double Y3 = -face_signum(bits, v2y, 2) * (double)u[yface_idx(d, xP, yO, zM)];
    double Y4 = face_signum(bits, v2y, 3) * (double)u[yface_idx(d, xP, yO + 1, zM)];
    double Y5 = -face_signum(bits, v3y, 2) * (double)u[yface_idx(d, xM, yO, zP)];
    double Y6 = face_signum(bits, v3y, 3) * (double)u[yface_idx(d, xM, yO + 1, zP)];
    double Y7 = -face_signum(bits, v4y, 2) * (double)u[yface_idx(d, xP, yO, zP)];
    double Y8 = face_signum(bits, v4y, 3) * (double)u[yface_idx(d, xP, yO + 1, zP)];

    double Z1 = face_signum(bits, v1z, 0) * (double)u[zface_idx(d, xM, yM, zO)];
    double Z2 = face_signum(bits, v3z, 0) * (double)u[zface_idx(d, xM, yP, zO)];
    double Z3 = face_signum(bits, v2z, 0) * (double)u[zface_idx(d, xP, yM, zO)];
    double Z4 = face_signum(bits, v4z, 0) * (double)u[zface_idx(d, xP, yP, zO)];
    double Z5 = -face_signum(bits, v1z, 1) * (double)u[zface_idx(d, xM, yM, zO + 1)];
    double Z6 = -face_signum(bits, v3z, 1) * (double)u[zface_idx(d, xM, yP, zO + 1)];
    double Z7 = -face_signum(bits, v2z, 1) * (double)u[zface_idx(d, xP, yM, zO + 1)];
    double Z8 = -face_signum(bits, v4z, 1) * (double)u[zface_idx(d, xP, yP, zO + 1)];

    double n[3], a, b, c0, c1;
    for (int q = 0; q < 3; ++q) n[q] = (p[q] - cfx[q]) * (1.0 / h);
    /* mix along y: (1,2) (3,4) (5,6) (7,8); then x: (.x,.y) (.z,.w); then z. */
    a = mixd(X1, X2, n[1]); b = mixd(X3, X4, n[1]);
    c0 = mixd(X5, X6, n[1]); c1 = mixd(X7, X8, n[1]);
    v[0] = mixd(mixd(a, b, n[0]), mixd(c0, c1, n[0]), n[2]);

    for (int q = 0; q < 3; ++q) n[q] = (p[q] - cfy[q]) * (1.0 / h);
    a = mixd(Y1, Y2, n[1]); b = mixd(Y3, Y4, n[1]);
    c0 = mixd(Y5, Y6, n[1]); c1 = mixd(Y7, Y8, n[1]);
    v[1] = mixd(mixd(a, b, n[0]), mixd(c0, c1, n[0]), n[2]);

    for (int q = 0; q < 3; ++q) n[q] = (p[q] - cfz[q]) * (1.0 / h);
    a = mixd(Z1, Z2, n[1]); b = mixd(Z3, Z4, n[1]);
    c0 = mixd(Z5, Z6, n[1]); c1 = mixd(Z7, Z8, n[1]);
    v[2] = mixd(mixd(a, b, n[0]), mixd(c0, c1, n[0]), n[2]);
}

/* Counter-based generator for respawns (SplitMix64 output function). */
uint32_t psfo_hash(uint64_t seed, uint64_t step, uint32_t idx, uint32_t k)
{
    uint64_t x = seed ^ (step * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)idx << 32) ^
                 ((uint64_t)k * 0xD1B54A32D192ED03ull);
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (uint32_t)(x >> 32);
}

static void clamp_box(const psfo_grid *g, double p[3])
{
    for (int c = 0; c < 3; ++c) p[c] = clampd(p[c], g->aabb_min[c], g->aabb_max[c]);
}

/*
 * Advance particles one step.  pos: [P][3] FP64 positions (kept in FP64
 * between steps), life: [P] float.  integrator: 1 = forward Euler (the
 * reference), 4 = classical RK4.
 */
void psfo_trace(const psfo_grid *g, const float *u, const uint32_t *bits, double *pos, float *life,
                int64_t P, double dt, int32_t integrator, float lifetime, uint64_t seed,
                uint64_t step)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < P; ++i) {
        double *p = pos + 3 * i;
        if (life[i] > 0.0f) {
            double v[3];
            if (integrator == 4) {
                double k1[3], k2[3], k3[3], k4[3], q[3];
                velocity_at(g, u, bits, p, k1);
                for (int c = 0; c < 3; ++c) q[c] = p[c] + 0.5 * dt * k1[c];
                clamp_box(g, q);
                velocity_at(g, u, bits, q, k2);
                for (int c = 0; c < 3; ++c) q[c] = p[c] + 0.5 * dt * k2[c];
                clamp_box(g, q);
                velocity_at(g, u, bits, q, k3);
                for (int c = 0; c < 3; ++c) q[c] = p[c] + dt * k3[c];
                clamp_box(g, q);
                velocity_at(g, u, bits, q, k4);
                for (int c = 0; c < 3; ++c) v[c] = (k1[c] + 2.0 * k2[c] + 2.0 * k3[c] + k4[c]) / 6.0;
            } else {
                velocity_at(g, u, bits, p, v);
            }
            for (int c = 0; c < 3; ++c) p[c] = p[c] + dt * v[c];
            clamp_box(g, p);
            life[i] = life[i] - 1.0f;
        } else {
            /* psfsolver.cpp:217-222 with a counter-based generator. */
            uint32_t r1 = psfo_hash(seed, step, (uint32_t)i, 1) % 1024u;
            uint32_t r2 = psfo_hash(seed, step, (uint32_t)i, 2) % 1024u;
            uint32_t r3 = psfo_hash(seed, step, (uint32_t)i, 3) % 1024u;
            float cz = g->aabb_min[2] + 0.5f * (g->aabb_max[2] - g->aabb_min[2]);
            p[0] = (double)(float)(((double)r1 / 1024.0 - 0.5) * 0.25);
            p[1] = (double)(g->aabb_min[1] + 0.2f);
            p[2] = (double)(float)(-(double)cz + ((double)r3 / 1024.0 - 0.5) * 0.25);
            life[i] = (float)((double)lifetime * ((double)r2 / 1024.0));
        }
    }
}
