/*
 * aster_oracle.c -- CPU restatement of the reference Aster force/integration
 * hot path, plus FP64 CPU references for the forms the reference lacks.
 *
 * TEST INFRASTRUCTURE ONLY. Used by tests/, the golden-fixture script and the
 * CPU-baseline leg of bench.py as the checker; never linked by the product.
 * Compiled with -ffp-contract=off (no FMA) so that every FP64/FP32 expression
 * rounds exactly as written; where the GPU must reproduce an integer or a
 * decision bit-exactly, the GPU code uses the same operation order with
 * explicitly rounded intrinsics.
 *
 * Pinned against the reference itself: tests/test_oracle.py compares each
 * function here with the reference CPU code compiled from its own sources
 * (oracle/_ref/libaster_ref.so) and with the committed golden fixtures.
 *
 * Functions and the reference code they restate:
 *   orc_pair_acc        src/physics/tool_chain_impl.cpp:65-137 (compute_gravitational: Newton
 *                       + get_pn1 + get_pn2 + get_pn25, CPU forms, as accelerations)
 *   orc_allpairs        src/utils/builder_endpoint.cpp:729-757 (Parallelized)
 *   orc_morton30        src/solvers/bh_specialization.cpp:30-46 (get_morton, part1by2)
 *   orc_morton30_compat include/Aster/kernels/morton_writer.cl.h:72-122 (gen_mortons 3-D)
 *   orc_sort_codes      src/solvers/barnes_hut.cpp:324 with a stable sort (ties by index)
 *   orc_karras          src/solvers/barnes_hut.cpp:338-396 (CPU, tie-break on sorted position)
 *                       include/Aster/kernels/BHH_specific.cl.h:171-272 (compat: body index)
 *   orc_bottom_up       src/solvers/barnes_hut.cpp:137-152 (NodesArray::unite) + new AABB/opening radius
 *   orc_lbvh_forces     new group-based traversal (same decisions as the GPU kernel)
 *   orc_node_velocities src/solvers/barnes_hut.cpp:150 (NodesArray::unite, velocities)
 *   orc_lbvh_forces_pn  the traversal with the pair law of compute_gravitational and node
 *                       velocities, as Barnes_Hut::get_node_body (barnes_hut.cpp:202-258)
 *   orc_kdk             src/physics/tool_chain_impl.cpp:169-185 restated as kick-drift-kick
 *                       with the acceleration cached across steps
 *   orc_saba            src/integrators/SABA.cpp:14-553 (update_SABA1..10, CPU forms;
 *                       SABA1 is update_euler, tool_chain_impl.cpp:158-167)
 *   orc_wh              Wisdom-Holman in democratic heliocentric coordinates (Wisdom &
 *                       Holman 1991; Duncan, Levison & Lee 1998), the published method
 *                       the reference's update_WH_planetary (tool_chain_impl.cpp:186-290,
 *                       WH_planetary.cl.h) aims at; its own step re-applies the central
 *                       force in the kick, so parity is with the published method
 *   orc_kepler          universal-variable Kepler drift (Stumpff functions, Laguerre-
 *                       Conway iteration)
 *   orc_saba_coeffs     the SABA_n drift/kick coefficients (Laskar & Robutel 2001):
 *                       Gauss-Legendre nodes and weights on [0,1], the values
 *                       include/Aster/physics/coeffs.h:8-161 tabulates
 *   orc_energy          Plummer-softened energy (the reference's collectors.cpp:19-53
 *                       uses -Gm_im_j/(r+softening); orc_energy_ref restates that too)
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define PN1_FLAG 0x10
#define PN2_FLAG 0x100
#define PN25_FLAG 0x1000
#define EIH_FLAG 0x10000

/* ------------------------------------------------------------------------ */
/* threading helper                                                          */
/* ------------------------------------------------------------------------ */
typedef void (*orc_range_fn)(void* ctx, long lo, long hi);
typedef struct { orc_range_fn fn; void* ctx; long n, chunk; long* next; pthread_mutex_t* mu; } orc_job;

static int g_threads = 0;
void orc_set_threads(int t) { g_threads = t; }
static int orc_threads(void) {
    if (g_threads > 0) return g_threads;
    const char* e = getenv("ASTER_ORACLE_THREADS");
    int v = e ? atoi(e) : 0;
    if (v <= 0) v = (int)sysconf(_SC_NPROCESSORS_ONLN);
    return v > 0 ? v : 1;
}

static void* orc_worker(void* arg) {
    orc_job* j = (orc_job*)arg;
    for (;;) {
        pthread_mutex_lock(j->mu);
        long lo = *j->next;
        *j->next += j->chunk;
        pthread_mutex_unlock(j->mu);
        if (lo >= j->n) break;
        long hi = lo + j->chunk < j->n ? lo + j->chunk : j->n;
        j->fn(j->ctx, lo, hi);
    }
    return NULL;
}

static void orc_parallel(long n, orc_range_fn fn, void* ctx) {
    int T = orc_threads();
    if (T > 256) T = 256;
    if (n <= 0) return;
    if (T == 1 || n < 64) { fn(ctx, 0, n); return; }
    long next = 0;
    pthread_mutex_t mu;
    pthread_mutex_init(&mu, NULL);
    orc_job job = {fn, ctx, n, n / (T * 16) > 0 ? n / (T * 16) : 1, &next, &mu};
    pthread_t th[256];
    for (int t = 1; t < T; ++t) pthread_create(&th[t], NULL, orc_worker, &job);
    orc_worker(&job);
    for (int t = 1; t < T; ++t) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&mu);
}

/* ------------------------------------------------------------------------ */
/* pair law                                                                  */
/* ------------------------------------------------------------------------ */
/* Acceleration on body 1 from body 2 (G, 1/c^2, softening = eps^2 added to r^2).
 * Newton: G m2 d / r^3 with d = p2 - p1, r^2 = d.d + eps2 (tool_chain_impl.cpp:121-127,
 * divided by m1 as Parallelized does). 1PN (tool_chain_impl.cpp:110-118) with
 * n = -(d/r) = (p1-p2)/r:
 *   a1 = G m2 / r^2 [ n(-v1^2 - 2 v2^2 + 4 v1.v2 + 1.5 (n.v2)^2 + 5 G m1/r + 4 G m2/r)
 *                     + (v1 - v2)(4 n.v1 - 3 n.v2) ] / c^2
 * (the reference multiplies by m1 to make a force and Parallelized divides it
 * back out, so the acceleration is a1 itself). */
/* Acceleration of body 1 (the reference's force divided by m1). inv_c = 1/c.
 * The post-Newtonian terms use n = (x1 - x2)/r (the reference passes -norm)
 * and are scaled by c^-2, c^-4, c^-5 as in compute_gravitational
 * (tool_chain_impl.cpp:120-137); get_pn2 (:79-107) and get_pn25 (:65-77) are
 * written out in the reference's operation order. */
void orc_pair_acc(double G, double inv_c, double eps2, int pn,
                  double m1, double m2, const double* v1, const double* v2,
                  const double* p1, const double* p2, double* a) {
    double d[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
    double inv_r = 1.0 / sqrt(r2);
    double inv_r2 = inv_r * inv_r;
    double s = G * m2 * inv_r2 * inv_r;
    a[0] = d[0] * s; a[1] = d[1] * s; a[2] = d[2] * s;
    if (!(pn & (PN1_FLAG | PN2_FLAG | PN25_FLAG))) return;
    double n[3] = {-d[0] * inv_r, -d[1] * inv_r, -d[2] * inv_r};
    double v1sq = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
    double v2sq = v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2];
    double v12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
    double nv1 = n[0] * v1[0] + n[1] * v1[1] + n[2] * v1[2];
    double nv2 = n[0] * v2[0] + n[1] * v2[1] + n[2] * v2[2];
    double inv_c2 = inv_c * inv_c;
    if (pn & PN1_FLAG) {
        double A = -v1sq - 2.0 * v2sq + 4.0 * v12 + 1.5 * nv2 * nv2 + 5.0 * G * m1 * inv_r + 4.0 * G * m2 * inv_r;
        double Bc = 4.0 * nv1 - 3.0 * nv2;
        double f = G * m2 * inv_r2 * inv_c2;
        for (int k = 0; k < 3; ++k) a[k] += (n[k] * A + (v1[k] - v2[k]) * Bc) * f;
    }
    if (pn & PN2_FLAG) {
        double nv22 = nv2 * nv2, nv12 = nv1 * nv1;
        double pn1 = G * m1 * inv_r, pn2 = G * m2 * inv_r;
        double Sn = -2 * v2sq * v2sq + 4 * v2sq * v12 - 2 * v12 * v12 + 3.0 / 2.0 * v1sq * nv22 +
                    9.0 / 2.0 * v2sq * nv22 - 6 * v12 * nv22 - 15.0 / 8.0 * nv22 * nv22 +
                    pn1 * (-15.0 / 4.0 * v1sq + 5.0 / 4.0 * v2sq - 5.0 / 2.0 * v12 + 39.0 / 2.0 * nv12 -
                           39.0 * nv1 * nv2 + 17.0 / 2.0 * nv22) +
                    pn2 * (4 * v2sq - 8 * v12 + 2 * nv12 - 4 * nv1 * nv2 - 6 * nv22);
        double Sv = v1sq * nv2 + 4 * v2sq * nv1 - 5 * v2sq * nv2 - 4 * v12 * nv1 + 4 * v12 * nv2 -
                    6 * nv1 * nv22 + 9.0 / 2.0 * nv22 * nv2 + pn1 * (-63.0 / 4.0 * nv1 + 55.0 / 4.0 * nv2) +
                    pn2 * (-2 * nv1 - 2 * nv2);
        double f = G * m2 * inv_r * inv_r;
        double g3 = G * G * G * m2 * inv_r * inv_r * inv_r * inv_r;
        double Sm = -57.0 / 4.0 * m1 * m1 - 9 * m2 * m2 - 69.0 / 2.0 * m1 * m2;
        double c4 = inv_c * inv_c * inv_c * inv_c;
        for (int k = 0; k < 3; ++k) a[k] += c4 * (f * (n[k] * Sn + (v1[k] - v2[k]) * Sv) + g3 * n[k] * Sm);
    }
    if (pn & PN25_FLAG) {
        double pn1 = G * m1 * inv_r, pn2 = G * m2 * inv_r;
        double dv[3] = {v1[0] - v2[0], v1[1] - v2[1], v1[2] - v2[2]};
        double sq = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
        double i1 = -sq + 2 * pn1 - 8 * pn2;
        double nd = nv1 - nv2;
        double i2 = 3 * sq - 6 * pn1 + 52.0 / 3.0 * pn2;
        double f = 4.0 / 5.0 * G * G * m1 * m2 * inv_r * inv_r * inv_r;
        double c5 = inv_c * inv_c * inv_c * inv_c * inv_c;
        for (int k = 0; k < 3; ++k) a[k] += c5 * ((dv[k] * i1 + n[k] * nd * i2) * f);
    }
}

typedef struct {
    long n, ns; const double *pos, *vel, *m; const long* targets;
    double G, inv_c, eps2; int pn; double* acc;
} allpairs_ctx;

static void allpairs_range(void* c_, long lo, long hi) {
    allpairs_ctx* c = (allpairs_ctx*)c_;
    for (long t = lo; t < hi; ++t) {
        long i = c->targets ? c->targets[t] : t;
        double ax = 0, ay = 0, az = 0, a[3];
        for (long j = 0; j < c->n; ++j) {
            if (j == i) continue;
            orc_pair_acc(c->G, c->inv_c, c->eps2, c->pn, c->m[i], c->m[j], c->vel + 3 * i, c->vel + 3 * j,
                         c->pos + 3 * i, c->pos + 3 * j, a);
            ax += a[0]; ay += a[1]; az += a[2];
        }
        c->acc[3 * t] = ax; c->acc[3 * t + 1] = ay; c->acc[3 * t + 2] = az;
    }
}

/* All-pairs accelerations (skip j == i). targets == NULL: every body, else the
 * nt listed bodies (acc has nt rows). vel may be NULL when pn has no PN bit. */
void orc_allpairs(long n, const double* pos, const double* vel, const double* m,
                  double G, double inv_c, double eps2, int pn,
                  long nt, const long* targets, double* acc) {
    double* vtmp = NULL;
    if (!vel) { vtmp = (double*)calloc((size_t)n * 3, sizeof(double)); vel = vtmp; }
    allpairs_ctx c = {n, nt, pos, vel, m, targets, G, inv_c, eps2, pn, acc};
    orc_parallel(targets ? nt : n, allpairs_range, &c);
    free(vtmp);
}

/* ------------------------------------------------------------------------ */
/* energy / momentum                                                         */
/* ------------------------------------------------------------------------ */
typedef struct { long n; const double *pos, *vel, *m; double G, eps2; int ref_form; double* part; } energy_ctx;

static void energy_range(void* c_, long lo, long hi) {
    energy_ctx* c = (energy_ctx*)c_;
    for (long i = lo; i < hi; ++i) {
        const double* v = c->vel + 3 * i;
        double e = 0.5 * c->m[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (long j = i + 1; j < c->n; ++j) {
            double dx = c->pos[3 * j] - c->pos[3 * i], dy = c->pos[3 * j + 1] - c->pos[3 * i + 1],
                   dz = c->pos[3 * j + 2] - c->pos[3 * i + 2];
            double r2 = dx * dx + dy * dy + dz * dz;
            double inv = c->ref_form ? 1.0 / (sqrt(r2) + c->eps2) : 1.0 / sqrt(r2 + c->eps2);
            e -= c->G * c->m[i] * c->m[j] * inv;
        }
        c->part[i] = e;
    }
}

/* Total energy. ref_form = 0: Plummer potential -G m_i m_j / sqrt(r^2 + eps2),
 * consistent with the softened force. ref_form = 1: the reference's
 * collectors.cpp:43 form -G m_i m_j / (r + softening) with softening = eps2. */
double orc_energy(long n, const double* pos, const double* vel, const double* m,
                  double G, double eps2, int ref_form) {
    double* part = (double*)malloc((size_t)n * sizeof(double));
    energy_ctx c = {n, pos, vel, m, G, eps2, ref_form, part};
    orc_parallel(n, energy_range, &c);
    double e = 0;
    for (long i = 0; i < n; ++i) e += part[i];
    free(part);
    return e;
}

void orc_momentum(long n, const double* vel, const double* m, double* p) {
    p[0] = p[1] = p[2] = 0;
    for (long i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) p[k] += m[i] * vel[3 * i + k];
}

/* ------------------------------------------------------------------------ */
/* integrators                                                               */
/* ------------------------------------------------------------------------ */
/* Kick-drift-kick leapfrog with the acceleration cached between steps:
 *   v += a dt/2; x += v dt; a = A(x); v += a dt/2
 * The reference's update_leapfrog (tool_chain_impl.cpp:169-185) is the same map
 * written as x += v dt + a dt^2/2, v += a dt/2, A(x), v += a dt/2 and evaluates
 * A twice per step; both produce the same trajectory up to rounding.
 * acc (n*3) must hold A(x0) on entry (computed here if acc_valid == 0);
 * acc_steps (nsteps*n*3, optional) receives A(x_{k+1}). */
void orc_kdk(long n, double* pos, double* vel, const double* m, double G, double inv_c,
             double eps2, int pn, double dt, int nsteps, double* acc, int acc_valid,
             double* acc_steps) {
    if (!acc_valid) orc_allpairs(n, pos, vel, m, G, inv_c, eps2, pn, 0, NULL, acc);
    const double h = 0.5 * dt;
    for (int k = 0; k < nsteps; ++k) {
        for (long i = 0; i < 3 * n; ++i) { vel[i] += acc[i] * h; pos[i] += vel[i] * dt; }
        orc_allpairs(n, pos, vel, m, G, inv_c, eps2, pn, 0, NULL, acc);
        for (long i = 0; i < 3 * n; ++i) vel[i] += acc[i] * h;
        if (acc_steps) memcpy(acc_steps + (size_t)k * n * 3, acc, (size_t)n * 3 * sizeof(double));
    }
}

/* ------------------------------------------------------------------------ */
/* SABA_n                                                                    */
/* ------------------------------------------------------------------------ */
/* SABA_n (n >= 2): drift c1, then for k = 1..n: forces, kick d_k, drift
 * c_{k+1}. With x_1 < ... < x_n the Gauss-Legendre nodes on [0,1] and w_k the
 * weights: c_1 = x_1, c_{k+1} = x_{k+1} - x_k, c_{n+1} = 1 - x_n, d_k = w_k.
 * Nodes by Newton's method on the Legendre recurrence in long double. Returns
 * the number of kicks; c_out gets n + 1 drifts, d_out n kicks. Order 1 is the
 * reference's SABA1 = update_euler: one kick of 1 followed by a drift of 1
 * (c_out = {0, 1}, d_out = {1}). */
int orc_saba_coeffs(int order, double* c_out, double* d_out) {
    if (order < 1 || order > 10) return -1;
    if (order == 1) { c_out[0] = 0.0; c_out[1] = 1.0; d_out[0] = 1.0; return 1; }
    const int n = order;
    long double x[10] = {0}, w[10] = {0};
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < n; ++i) {
        long double z = cosl(pi * (i + 0.75L) / (n + 0.5L)), dp = 1.0L;
        for (int it = 0; it < 100; ++it) {
            long double p0 = 1.0L, p1 = z;
            for (int k = 2; k <= n; ++k) {
                long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0L);
            long double dz = p1 / dp;
            z -= dz;
            if (fabsl(dz) < 1e-19L) break;
        }
        {
            long double p0 = 1.0L, p1 = z;
            for (int k = 2; k <= n; ++k) {
                long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0L);
        }
        /* i = 0 is the largest root: store ascending on [0,1] */
        x[n - 1 - i] = 0.5L * (1.0L + z);
        w[n - 1 - i] = 1.0L / ((1.0L - z * z) * dp * dp);
    }
    c_out[0] = (double)x[0];
    for (int k = 1; k < n; ++k) c_out[k] = (double)(x[k] - x[k - 1]);
    c_out[n] = (double)(1.0L - x[n - 1]);
    for (int k = 0; k < n; ++k) d_out[k] = (double)w[k];
    return n;
}

/* nsteps of a drift/kick sequence with all-pairs forces: drift c[0], then for
 * k = 0..nk-1: forces, kick d[k], drift c[k+1] (the form of every
 * update_SABAn for n >= 2, SABA.cpp:19-553). */
void orc_saba_seq(long n, double* pos, double* vel, const double* m, double G, double inv_c, double eps2, int pn,
                  double dt, int nk, const double* c, const double* d, int nsteps, double* acc) {
    for (int s = 0; s < nsteps; ++s) {
        for (long i = 0; i < 3 * n; ++i) pos[i] += vel[i] * c[0] * dt;
        for (int k = 0; k < nk; ++k) {
            orc_allpairs(n, pos, vel, m, G, inv_c, eps2, pn, 0, NULL, acc);
            for (long i = 0; i < 3 * n; ++i) {
                vel[i] += acc[i] * d[k] * dt;
                pos[i] += vel[i] * c[k + 1] * dt;
            }
        }
    }
}

/* nsteps of SABA_order with all-pairs forces. Order 1 is the reference's
 * update_euler (forces, v += a dt, x += v dt). */
void orc_saba(long n, double* pos, double* vel, const double* m, double G, double inv_c, double eps2, int pn,
              double dt, int order, int nsteps, double* acc) {
    double c[11], d[10];
    const int nk = orc_saba_coeffs(order, c, d);
    if (nk < 0) return;
    if (order > 1) {
        orc_saba_seq(n, pos, vel, m, G, inv_c, eps2, pn, dt, nk, c, d, nsteps, acc);
        return;
    }
    for (int s = 0; s < nsteps; ++s) {
        orc_allpairs(n, pos, vel, m, G, inv_c, eps2, pn, 0, NULL, acc);
        for (long i = 0; i < 3 * n; ++i) { vel[i] += acc[i] * dt; pos[i] += vel[i] * dt; }
    }
}

/* ------------------------------------------------------------------------ */
/* Wisdom-Holman (democratic heliocentric)                                  */
/* ------------------------------------------------------------------------ */
/* Stumpff functions c2(z) = (1 - cos sqrt z)/z and c3(z) = (sqrt z - sin sqrt z)/
 * sqrt(z)^3 (hyperbolic forms for z < 0), by their power series near 0. */
static void orc_stumpff(double z, double* c2, double* c3) {
    if (fabs(z) < 0.5) {
        double t2 = 0.5, t3 = 1.0 / 6.0, s2 = 0.0, s3 = 0.0;
        for (int k = 1; k <= 10; ++k) {
            s2 += t2;
            s3 += t3;
            t2 *= -z / ((2.0 * k + 1.0) * (2.0 * k + 2.0));
            t3 *= -z / ((2.0 * k + 2.0) * (2.0 * k + 3.0));
        }
        *c2 = s2;
        *c3 = s3;
    } else if (z > 0.0) {
        double s = sqrt(z), h = sin(0.5 * s);
        *c2 = 2.0 * h * h / z;
        *c3 = (s - sin(s)) / (z * s);
    } else {
        double s = sqrt(-z);
        *c2 = (cosh(s) - 1.0) / (-z);
        *c3 = (sinh(s) - s) / (-z * s);
    }
}

/* Advances the relative state (r, v) along its Kepler orbit about mu for dt.
 * Universal anomaly chi solves sqrt(mu) dt = r0 chi + s0 chi^2 c2 + (1 - a r0)
 * chi^3 c3 (s0 = r.v / sqrt mu, a = 2/r0 - v^2/mu, z = a chi^2), by
 * Laguerre-Conway steps from chi = sqrt(mu) dt / r0; then the f and g
 * functions. Returns 0, or -1 (state unchanged) for r = 0 or no convergence. */
int orc_kepler(double* r, double* v, double mu, double dt) {
    const double r0 = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (!(r0 > 0.0) || !(mu > 0.0)) return -1;
    if (dt == 0.0) return 0;
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double smu = sqrt(mu);
    const double s0 = (r[0] * v[0] + r[1] * v[1] + r[2] * v[2]) / smu;
    const double a = 2.0 / r0 - v2 / mu;
    const double b = 1.0 - a * r0;
    double chi = smu * dt / r0, c2 = 0.5, c3 = 1.0 / 6.0;
    int ok = 0;
    for (int it = 0; it < 64; ++it) {
        const double z = a * chi * chi;
        orc_stumpff(z, &c2, &c3);
        const double F = r0 * chi + s0 * chi * chi * c2 + b * chi * chi * chi * c3 - smu * dt;
        const double Fp = r0 + s0 * chi * (1.0 - z * c3) + b * chi * chi * c2;
        const double Fpp = s0 * (1.0 - z * c2) + b * chi * (1.0 - z * c3);
        const double disc = fabs(16.0 * Fp * Fp - 20.0 * F * Fpp);
        const double den = Fp + (Fp >= 0.0 ? 1.0 : -1.0) * sqrt(disc);
        const double d = den != 0.0 ? 5.0 * F / den : F / Fp;
        chi -= d;
        if (fabs(d) <= 1e-15 * (1.0 + fabs(chi))) { ok = 1; break; }
    }
    if (!ok || !isfinite(chi)) return -1;
    const double z = a * chi * chi;
    orc_stumpff(z, &c2, &c3);
    const double f = 1.0 - chi * chi * c2 / r0;
    const double g = dt - chi * chi * chi * c3 / smu;
    double rn[3];
    for (int k = 0; k < 3; ++k) rn[k] = f * r[k] + g * v[k];
    const double rr = sqrt(rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2]);
    const double fd = smu / (rr * r0) * chi * (z * c3 - 1.0);
    const double gd = 1.0 - chi * chi * c2 / rr;
    for (int k = 0; k < 3; ++k) {
        const double vn = fd * r[k] + gd * v[k];
        r[k] = rn[k];
        v[k] = vn;
    }
    return 0;
}

/* Interaction acceleration among bodies 1..n-1 (body 0 excluded as source
 * and target): Newtonian, softened, from heliocentric positions Q. */
static void orc_wh_interaction(long n, const double* Q, const double* m, double G, double eps2, double* a) {
    memset(a, 0, (size_t)n * 3 * sizeof(double));
    for (long i = 1; i < n; ++i)
        for (long j = 1; j < n; ++j) {
            if (j == i) continue;
            double d[3] = {Q[3 * j] - Q[3 * i], Q[3 * j + 1] - Q[3 * i + 1], Q[3 * j + 2] - Q[3 * i + 2]};
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
            double inv = 1.0 / sqrt(r2);
            double s = G * m[j] * inv * inv * inv;
            for (int k = 0; k < 3; ++k) a[3 * i + k] += d[k] * s;
        }
}

/* nsteps of Wisdom-Holman with body 0 as the central mass, in democratic
 * heliocentric coordinates: Q_i = x_i - x_0, V_i = v_i - v_cm (i >= 1).
 * H = sum_i (V_i^2/2 - G m_0/|Q_i|) m_i  [Kepler, A]
 *   - sum_{1<=i<j} G m_i m_j / |Q_i - Q_j|  [interaction, B]
 *   + |sum_i m_i V_i|^2 / (2 m_0)  [linear drift of the centre, C].
 * One step: C(dt/2) B(dt/2) A(dt) C(dt/2) B(dt/2) (B and C commute: the
 * interaction kick does not change sum_i m_i V_i, and the linear drift moves
 * every Q_i alike, so the interaction of the step's end is the next step's). The
 * barycentre moves uniformly; the inertial state is rebuilt at the end.
 * Returns 0 or -1 (a Kepler drift failed). */
int orc_wh(long n, double* pos, double* vel, const double* m, double G, double eps2, double dt, int nsteps) {
    if (n < 2 || !(m[0] > 0.0)) return -1;
    double M = 0.0, xc[3] = {0, 0, 0}, vc[3] = {0, 0, 0};
    for (long i = 0; i < n; ++i) {
        M += m[i];
        for (int k = 0; k < 3; ++k) { xc[k] += m[i] * pos[3 * i + k]; vc[k] += m[i] * vel[3 * i + k]; }
    }
    for (int k = 0; k < 3; ++k) { xc[k] /= M; vc[k] /= M; }
    double* Q = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* V = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* a = (double*)malloc((size_t)n * 3 * sizeof(double));
    for (long i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            Q[3 * i + k] = i ? pos[3 * i + k] - pos[k] : 0.0;
            V[3 * i + k] = i ? vel[3 * i + k] - vc[k] : 0.0;
        }
    const double mu = G * m[0], h = 0.5 * dt;
    int st = 0;
    orc_wh_interaction(n, Q, m, G, eps2, a);
    for (int s = 0; s < nsteps && st == 0; ++s) {
        double P[3] = {0, 0, 0};
        /* C(h), B(h) with the cached interaction, A(dt) */
        for (long i = 1; i < n; ++i)
            for (int k = 0; k < 3; ++k) P[k] += m[i] * V[3 * i + k];
        for (long i = 1; i < n; ++i) {
            for (int k = 0; k < 3; ++k) {
                Q[3 * i + k] += P[k] / m[0] * h;
                V[3 * i + k] += a[3 * i + k] * h;
            }
            if (orc_kepler(Q + 3 * i, V + 3 * i, mu, dt) != 0) st = -1;
        }
        /* C(h), then B(h) with the interaction at the new positions */
        P[0] = P[1] = P[2] = 0.0;
        for (long i = 1; i < n; ++i)
            for (int k = 0; k < 3; ++k) P[k] += m[i] * V[3 * i + k];
        for (long i = 1; i < n; ++i)
            for (int k = 0; k < 3; ++k) Q[3 * i + k] += P[k] / m[0] * h;
        orc_wh_interaction(n, Q, m, G, eps2, a);
        for (long i = 1; i < n; ++i)
            for (int k = 0; k < 3; ++k) V[3 * i + k] += a[3 * i + k] * h;
    }
    /* inertial state: barycentre at xc + vc t */
    double T = dt * nsteps, S[3] = {0, 0, 0}, P[3] = {0, 0, 0};
    for (long i = 1; i < n; ++i)
        for (int k = 0; k < 3; ++k) { S[k] += m[i] * Q[3 * i + k]; P[k] += m[i] * V[3 * i + k]; }
    double x0[3];
    for (int k = 0; k < 3; ++k) x0[k] = xc[k] + vc[k] * T - S[k] / M;
    for (int k = 0; k < 3; ++k) { pos[k] = x0[k]; vel[k] = vc[k] - P[k] / m[0]; }
    for (long i = 1; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            pos[3 * i + k] = x0[k] + Q[3 * i + k];
            vel[3 * i + k] = vc[k] + V[3 * i + k];
        }
    free(Q); free(V); free(a);
    return st;
}

/* ------------------------------------------------------------------------ */
/* Morton codes                                                              */
/* ------------------------------------------------------------------------ */
static uint32_t part1by2_32(uint32_t n) {
    n = (n | (n << 16)) & 0x030000FFu;
    n = (n | (n << 8)) & 0x0300F00Fu;
    n = (n | (n << 4)) & 0x030C30C3u;
    n = (n | (n << 2)) & 0x09249249u;
    return n;
}

static uint64_t part1by2_64(uint64_t n) {
    n &= 0x1FFFFFull;
    n = (n | (n << 32)) & 0x001F00000000FFFFull;
    n = (n | (n << 16)) & 0x001F0000FF0000FFull;
    n = (n | (n << 8)) & 0x100F00F00F00F00Full;
    n = (n | (n << 4)) & 0x10C30C30C30C30C3ull;
    n = (n | (n << 2)) & 0x1249249249249249ull;
    return n;
}

/* Reference get_morton: x' = (x + B)/(2B), ix = min((uint32)(x' * 1024), 1023),
 * code = part(iz)<<2 | part(iy)<<1 | part(ix). A negative x' is undefined
 * behaviour in the reference; with B = max |coord| it cannot occur, and this
 * restatement clamps it to 0. */
static uint32_t quant(double x, double B, double scale, uint32_t maxv) {
    double t = (x + B) / (2.0 * B);
    double s = t * scale;
    if (!(s > 0.0)) return 0;                 /* negative or NaN */
    if (s >= 4294967296.0) return maxv;
    uint32_t q = (uint32_t)s;
    return q < maxv ? q : maxv;
}

void orc_morton30(long n, const double* pos, double B, uint32_t* codes) {
    for (long i = 0; i < n; ++i) {
        uint32_t ix = quant(pos[3 * i], B, 1024.0, 1023u);
        uint32_t iy = quant(pos[3 * i + 1], B, 1024.0, 1023u);
        uint32_t iz = quant(pos[3 * i + 2], B, 1024.0, 1023u);
        codes[i] = (part1by2_32(iz) << 2) | (part1by2_32(iy) << 1) | part1by2_32(ix);
    }
}

/* 63-bit variant: 21 bits per axis, x' * 2^21 clamped to 2^21 - 1. */
void orc_morton63(long n, const double* pos, double B, uint64_t* codes) {
    for (long i = 0; i < n; ++i) {
        uint64_t ix = quant(pos[3 * i], B, 2097152.0, 2097151u);
        uint64_t iy = quant(pos[3 * i + 1], B, 2097152.0, 2097151u);
        uint64_t iz = quant(pos[3 * i + 2], B, 2097152.0, 2097151u);
        codes[i] = (part1by2_64(iz) << 2) | (part1by2_64(iy) << 1) | part1by2_64(ix);
    }
}

/* OpenCL gen_mortons (morton_writer.cl.h:72-122): clamp x' to [0,1], then
 * min((uint)(x'*1024), 1024), truncate to 16 bits and expand with the 10-bit
 * mask, so 1024 (a coordinate exactly at +B) becomes 0 on that axis. */
void orc_morton30_compat(long n, const double* pos, double B, uint32_t* codes) {
    for (long i = 0; i < n; ++i) {
        uint32_t q[3];
        for (int k = 0; k < 3; ++k) {
            double t = (pos[3 * i + k] + B) / (2.0 * B);
            t = fmin(fmax(t, 0.0), 1.0);
            uint32_t v = (uint32_t)(t * 1024.0);
            v = v < 1024u ? v : 1024u;
            q[k] = (uint32_t)(uint16_t)v;
        }
        codes[i] = part1by2_32(q[0]) | (part1by2_32(q[1]) << 1) | (part1by2_32(q[2]) << 2);
    }
}

/* ------------------------------------------------------------------------ */
/* sort                                                                      */
/* ------------------------------------------------------------------------ */
/* Stable LSD radix sort of (code, index): sorted codes + permutation
 * (perm[k] = input index of the k-th smallest). bits = 30 or 63.
 * descending != 0 reproduces the OpenCL bitonic order (radix.cl.h:11-13,26-91):
 * descending by (code, index). */
void orc_sort_codes(long n, const uint64_t* codes, int bits, int descending,
                    uint64_t* sorted, int32_t* perm) {
    uint64_t* k0 = (uint64_t*)malloc((size_t)n * 8);
    uint64_t* k1 = (uint64_t*)malloc((size_t)n * 8);
    int32_t* p0 = (int32_t*)malloc((size_t)n * 4);
    int32_t* p1 = (int32_t*)malloc((size_t)n * 4);
    for (long i = 0; i < n; ++i) { k0[i] = codes[i]; p0[i] = (int32_t)i; }
    for (int shift = 0; shift < bits; shift += 8) {
        long cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (long i = 0; i < n; ++i) cnt[((k0[i] >> shift) & 0xFF) + 1]++;
        for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
        for (long i = 0; i < n; ++i) {
            long d = cnt[(k0[i] >> shift) & 0xFF]++;
            k1[d] = k0[i]; p1[d] = p0[i];
        }
        uint64_t* tk = k0; k0 = k1; k1 = tk;
        int32_t* tp = p0; p0 = p1; p1 = tp;
    }
    for (long i = 0; i < n; ++i) {
        long s = descending ? n - 1 - i : i;
        sorted[i] = k0[s]; perm[i] = p0[s];
    }
    free(k0); free(k1); free(p0); free(p1);
}

/* ------------------------------------------------------------------------ */
/* Karras radix tree                                                         */
/* ------------------------------------------------------------------------ */
static int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }
static int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }

typedef struct { long n; const uint64_t* codes; const int32_t* perm; int bits; int compat; } karras_in;

/* delta(i,j): common-prefix length of sorted keys i and j; equal codes fall
 * back to key_bits + clz of the tie-break value: the sorted positions i^j (CPU,
 * barnes_hut.cpp:333-338) or the body indices (compat, BHH_specific.cl.h:180-189).
 * 30-bit codes use 32-bit clz as the reference does; 63-bit codes use 64-bit
 * clz and 64 + clz32 of the tie-break. Out-of-range j gives -1. */
static int kdelta(const karras_in* k, long i, long j) {
    if (j < 0 || j >= k->n) return -1;
    uint64_t a = k->codes[i], b = k->codes[j];
    if (a == b) {
        uint32_t t = k->compat ? (uint32_t)(k->perm[i] ^ k->perm[j]) : (uint32_t)(i ^ j);
        return (k->bits > 32 ? 64 : 32) + clz32(t);
    }
    return k->bits > 32 ? clz64(a ^ b) : clz32((uint32_t)(a ^ b));
}

/* Karras (2012) build. Nodes 0..n-1 are leaves in sorted order, n..2n-2 are
 * internal (internal i is node n+i), root = n, -1 = no child. Also emits
 * parent[2n-1] (parent[root] = -1) and the sorted-leaf range [lo, hi] of each
 * internal node (leaves: [k, k]). */
void orc_karras(long n, const uint64_t* sorted_codes, const int32_t* perm, int bits, int compat,
                int32_t* left, int32_t* right, int32_t* parent, int32_t* rlo, int32_t* rhi) {
    karras_in k = {n, sorted_codes, perm, bits, compat};
    for (long i = 0; i < 2 * n - 1; ++i) {
        left[i] = -1; right[i] = -1; parent[i] = -1;
        rlo[i] = (int32_t)(i < n ? i : -1); rhi[i] = (int32_t)(i < n ? i : -1);
    }
    for (long i = 0; i < n - 1; ++i) {
        int dl = (i == 0) ? -1 : kdelta(&k, i, i - 1);
        int dr = kdelta(&k, i, i + 1);
        int d = dr > dl ? 1 : -1;
        int dmin = d == 1 ? dl : dr;
        long lmax = 2;
        while (kdelta(&k, i, i + lmax * d) > dmin) lmax *= 2;
        long l = 0;
        for (long t = lmax / 2; t >= 1; t /= 2)
            if (kdelta(&k, i, i + (l + t) * d) > dmin) l += t;
        long j = i + l * d;
        int dnode = kdelta(&k, i, j);
        long s = 0;
        long range = j > i ? j - i : i - j;
        for (long t = (range + 1) / 2; t >= 1; t = (t + 1) / 2) {
            if (kdelta(&k, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        long gamma = i + s * d + (d < 0 ? d : 0);
        long lo = i < j ? i : j, hi = i < j ? j : i;
        long node = n + i;
        left[node] = (int32_t)(lo == gamma ? gamma : n + gamma);
        right[node] = (int32_t)(hi == gamma + 1 ? gamma + 1 : n + gamma + 1);
        parent[left[node]] = (int32_t)node;
        parent[right[node]] = (int32_t)node;
        rlo[node] = (int32_t)lo; rhi[node] = (int32_t)hi;
    }
}

/* ------------------------------------------------------------------------ */
/* bottom-up moments, bounds, opening radius                                 */
/* ------------------------------------------------------------------------ */
/* double -> float rounded down / up (exact emulation of the CUDA __double2float_rd/ru). */
static float f_rd(double d) { float f = (float)d; if ((double)f > d) f = nextafterf(f, -INFINITY); return f; }
static float f_ru(double d) { float f = (float)d; if ((double)f < d) f = nextafterf(f, INFINITY); return f; }

/* Node moments in FP64 exactly as NodesArray::unite (barnes_hut.cpp:137-152):
 *   M = m_R + m_L; c = (c_R m_R + c_L m_L) / M   (component-wise, this order)
 * except for a node without mass (M <= 0), which unite leaves with whatever
 * the array held before: here c = (c_R + c_L) / 2 (finite; the node adds
 * nothing to any force, and its ancestors' centres stay finite)
 * plus (new) the node AABB in FP32 (leaf: position rounded outwards; internal:
 * union of the children) and the squared opening radius
 *   r_crit = l/theta + |c - box_centre|, l = longest AABB side,
 * all in FP64, stored as a float rounded up (leaves: 0). */
void orc_bottom_up(long n, const int32_t* left, const int32_t* right, const int32_t* perm,
                   const double* pos, const double* m, double theta,
                   double* node_mass, double* node_com, float* bmin, float* bmax, float* rcrit2) {
    for (long k = 0; k < n; ++k) {
        long b = perm[k];
        node_mass[k] = m[b];
        for (int a = 0; a < 3; ++a) {
            node_com[3 * k + a] = pos[3 * b + a];
            bmin[3 * k + a] = f_rd(pos[3 * b + a]);
            bmax[3 * k + a] = f_ru(pos[3 * b + a]);
        }
        rcrit2[k] = 0.0f;
    }
    if (n < 2) return;
    /* post-order over internal nodes, iterative */
    long total = 2 * n - 1;
    int32_t* stack = (int32_t*)malloc((size_t)total * 4);
    char* done = (char*)calloc((size_t)total, 1);
    long sp = 0;
    stack[sp++] = (int32_t)n;
    while (sp > 0) {
        int32_t v = stack[sp - 1];
        int32_t L = left[v], R = right[v];
        if (v >= n && (!done[L] && L >= n)) { stack[sp++] = L; continue; }
        if (v >= n && (!done[R] && R >= n)) { stack[sp++] = R; continue; }
        sp--;
        if (v < n) { done[v] = 1; continue; }
        double M = node_mass[R] + node_mass[L];
        node_mass[v] = M;
        double lmax = 0.0, ctr[3];
        for (int a = 0; a < 3; ++a) {
            node_com[3 * v + a] = M > 0.0
                ? (node_com[3 * R + a] * node_mass[R] + node_com[3 * L + a] * node_mass[L]) / M
                : 0.5 * (node_com[3 * R + a] + node_com[3 * L + a]);
            bmin[3 * v + a] = fminf(bmin[3 * L + a], bmin[3 * R + a]);
            bmax[3 * v + a] = fmaxf(bmax[3 * L + a], bmax[3 * R + a]);
            double ext = (double)bmax[3 * v + a] - (double)bmin[3 * v + a];
            if (ext > lmax) lmax = ext;
            ctr[a] = 0.5 * ((double)bmin[3 * v + a] + (double)bmax[3 * v + a]);
        }
        double dx = node_com[3 * v] - ctr[0], dy = node_com[3 * v + 1] - ctr[1], dz = node_com[3 * v + 2] - ctr[2];
        double delta = sqrt(dx * dx + dy * dy + dz * dz);
        double rc = lmax / theta + delta;
        rcrit2[v] = f_ru(rc * rc);
        done[v] = 1;
    }
    free(stack);
    free(done);
}

/* ------------------------------------------------------------------------ */
/* group-based traversal                                                     */
/* ------------------------------------------------------------------------ */
/* Groups: the GPU walks the tree once per group (one warp). A group is a tree
 * node whose subtree holds at most GROUP leaves while its parent's holds more
 * (the root when n <= GROUP): a contiguous run of sorted leaves sharing a Morton
 * prefix, hence spatially compact. orc_groups lists them as (first sorted
 * leaf, count), ordered by first leaf.
 *
 * Walk: a node is opened for the whole group unless it is a leaf or the
 * squared distance from its FP32 centre of mass to the group's FP32 box exceeds
 * rcrit2; accepted nodes go to the group's interaction list. Decision
 * arithmetic is FP32, round-to-nearest, no FMA, in this exact order:
 *   d_a = max(0, max(glo_a - c_a, c_a - ghi_a)); d2 = (dx*dx + dy*dy) + dz*dz
 * where c = (float)com and the group box is the min/max of (float)pos.
 * Every body of the group then sums the list in FP64 (G m d / (d.d+eps2)^1.5,
 * zero when d.d+eps2 == 0). count[b] = list length of body b's group. */
#define ORC_GROUP 64

long orc_groups(long n, int group, const int32_t* parent, const int32_t* rlo, const int32_t* rhi,
                int32_t* start, int32_t* count) {
    if (n == 1) { start[0] = 0; count[0] = 1; return 1; }
    int32_t* at = (int32_t*)calloc((size_t)n, 4);  /* group size by first leaf */
    for (long v = 0; v < 2 * n - 1; ++v) {
        long sz = rhi[v] - rlo[v] + 1;
        if (sz > group) continue;
        long p = parent[v];
        if (p >= 0 && rhi[p] - rlo[p] + 1 <= group) continue;
        at[rlo[v]] = (int32_t)sz;
    }
    long ng = 0;
    for (long k = 0; k < n; ++k)
        if (at[k]) { start[ng] = (int32_t)k; count[ng] = at[k]; ++ng; }
    free(at);
    return ng;
}

typedef struct {
    long n; const int32_t *gstart, *gcount; const int32_t *left, *right, *perm; const double *pos, *node_mass,
        *node_com;
    const float* rcrit2; double G, eps2; double* acc; int32_t* count;
    /* post-Newtonian walk (pn has a PN bit): body velocities (input order),
     * node velocities (node order), 1/c */
    const double *vel, *node_vel; double inv_c; int pn;
} trav_ctx;

static void trav_range(void* c_, long glo, long ghi) {
    trav_ctx* c = (trav_ctx*)c_;
    long total = 2 * c->n - 1;
    int32_t* stack = (int32_t*)malloc((size_t)(total + 2) * 4);
    int32_t* list = (int32_t*)malloc((size_t)(total + 2) * 4);
    for (long g = glo; g < ghi; ++g) {
        long b0 = c->gstart[g], b1 = b0 + c->gcount[g];
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (long k = b0; k < b1; ++k)
            for (int a = 0; a < 3; ++a) {
                float p = (float)c->pos[3 * c->perm[k] + a];
                lo[a] = fminf(lo[a], p); hi[a] = fmaxf(hi[a], p);
            }
        long sp = 0, nl = 0;
        stack[sp++] = c->n >= 2 ? (int32_t)c->n : 0;
        while (sp > 0) {
            int32_t v = stack[--sp];
            if (v < c->n) { list[nl++] = v; continue; }
            float d[3];
            for (int a = 0; a < 3; ++a) {
                float cf = (float)c->node_com[3 * v + a];
                float u = lo[a] - cf, w = cf - hi[a];
                float t = u > w ? u : w;
                d[a] = t > 0.0f ? t : 0.0f;
            }
            float d2 = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
            if (d2 > c->rcrit2[v]) { list[nl++] = v; continue; }
            stack[sp++] = c->right[v];
            stack[sp++] = c->left[v];
        }
        for (long k = b0; k < b1; ++k) {
            long b = c->perm[k];
            if (c->count) c->count[b] = (int32_t)nl;
            const double* x = c->pos + 3 * b;
            double ax = 0, ay = 0, az = 0;
            if (c->pn & (PN1_FLAG | PN2_FLAG | PN25_FLAG)) {
                /* the reference pair law with the node's mass-weighted velocity
                 * (Barnes_Hut::get_node_body, barnes_hut.cpp:232-239) */
                for (long e = 0; e < nl; ++e) {
                    int32_t v = list[e];
                    const double* y = c->node_com + 3 * v;
                    double dx = y[0] - x[0], dy = y[1] - x[1], dz = y[2] - x[2];
                    if (dx * dx + dy * dy + dz * dz + c->eps2 == 0.0) continue;
                    double a[3];
                    orc_pair_acc(c->G, c->inv_c, c->eps2, c->pn, c->node_mass[k], c->node_mass[v], c->vel + 3 * b,
                                 c->node_vel + 3 * v, x, y, a);
                    ax += a[0]; ay += a[1]; az += a[2];
                }
                c->acc[3 * b] = ax; c->acc[3 * b + 1] = ay; c->acc[3 * b + 2] = az;
                continue;
            }
            for (long e = 0; e < nl; ++e) {
                int32_t v = list[e];
                const double* y = c->node_com + 3 * v;
                double dx = y[0] - x[0], dy = y[1] - x[1], dz = y[2] - x[2];
                double r2 = dx * dx + dy * dy + dz * dz + c->eps2;
                if (r2 == 0.0) continue;
                double inv = 1.0 / sqrt(r2);
                double s = c->node_mass[v] * inv * inv * inv;
                ax += dx * s; ay += dy * s; az += dz * s;
            }
            c->acc[3 * b] = c->G * ax; c->acc[3 * b + 1] = c->G * ay; c->acc[3 * b + 2] = c->G * az;
        }
    }
    free(stack);
    free(list);
}

/* ------------------------------------------------------------------------ */
/* batched ensemble: drift-kick compositions with the pairwise 1PN pair law  */
/* ------------------------------------------------------------------------ */
/* Yoshida (1990) fourth-order triple jump of the drift-kick-drift leapfrog:
 *   w1 = 1/(2 - 2^(1/3)), w0 = -2^(1/3)/(2 - 2^(1/3))
 *   drifts c = {w1/2, (w0+w1)/2, (w0+w1)/2, w1/2}, kicks d = {w1, w0, w1}
 * Leapfrog (integrator 0): c = {1/2, 1/2}, d = {1}. One step:
 *   x += c0 v dt; v += d0 a(x, v) dt; x += c1 v dt; ... ; x += c_last v dt
 * The acceleration is the reference pair law (orc_pair_acc, Newton + optional
 * pairwise 1PN of tool_chain_impl.cpp:110-137) summed over the system,
 * evaluated with the current (x, v). The reference has no Yoshida integrator
 * and no batched systems; this is the FP64 CPU reference for both. */
void orc_ens_coeffs(int integrator, double* c, double* d, int* nstages) {
    if (integrator == 1) {
        double cb = cbrt(2.0);
        double w1 = 1.0 / (2.0 - cb), w0 = -cb / (2.0 - cb);
        c[0] = c[3] = 0.5 * w1;
        c[1] = c[2] = 0.5 * (w0 + w1);
        d[0] = d[2] = w1;
        d[1] = w0;
        *nstages = 3;
    } else {
        c[0] = c[1] = 0.5;
        d[0] = 1.0;
        *nstages = 1;
    }
}

/* N-body 1PN accelerations of one system (n <= 64 bodies) in the
 * Einstein-Infeld-Hoffmann form (Einstein, Infeld & Hoffmann 1938; as written
 * in Will, Theory and Experiment in Gravitational Physics, 1993, sec. 6.2, and
 * Poisson & Will, Gravity, 2014, sec. 9.3), the accelerations of the other
 * bodies inside the 1PN terms taken at Newtonian order. With
 * r_ab = sqrt(|x_a - x_b|^2 + eps2), n_ab = (x_a - x_b)/r_ab,
 * phi_a = sum_{c != a} G m_c / r_ac and A_b the Newtonian acceleration of b:
 *   a_a = sum_{b != a} G m_b / r_ab^2 (-n_ab) [1 + (1/c^2)(-4 phi_a - phi_b + v_a^2 + 2 v_b^2
 *           - 4 v_a.v_b - 3/2 (n_ab.v_b)^2 + 1/2 (x_b - x_a).A_b)]
 *       + (1/c^2) sum_{b != a} G m_b / r_ab^2 [n_ab.(4 v_a - 3 v_b)] (v_a - v_b)
 *       + (7/(2 c^2)) sum_{b != a} G m_b A_b / r_ab
 * Sources at zero separation (the body itself, or one at exactly its
 * position) are left out of every sum, softened or not.
 * For two unsoftened bodies this is the pairwise law of get_pn1
 * (tool_chain_impl.cpp:110-118): the A_b terms give the 5 G m_a / r of its
 * bracket (1 from phi_b, 1/2 from (x_b - x_a).A_b, 7/2 from the last sum).
 * Beyond two bodies it adds the three-body couplings that get_pn1 omits. */
static void ens_eih_acc(long n, const double* x, const double* v, const double* m, double G, double inv_c2,
                        double eps2, double* acc) {
    double phi[64], an[64 * 3];
    for (long a = 0; a < n; ++a) {
        double p = 0, ax = 0, ay = 0, az = 0;
        for (long b = 0; b < n; ++b) {
            if (b == a) continue;
            double d[3] = {x[3 * b] - x[3 * a], x[3 * b + 1] - x[3 * a + 1], x[3 * b + 2] - x[3 * a + 2]};
            double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (d2 == 0.0) continue;
            double inv = 1.0 / sqrt(d2 + eps2);
            p += G * m[b] * inv;
            double s = G * m[b] * inv * inv * inv;
            ax += d[0] * s; ay += d[1] * s; az += d[2] * s;
        }
        phi[a] = p;
        an[3 * a] = ax; an[3 * a + 1] = ay; an[3 * a + 2] = az;
    }
    for (long a = 0; a < n; ++a) {
        const double* va = v + 3 * a;
        double va2 = va[0] * va[0] + va[1] * va[1] + va[2] * va[2];
        double pn[3] = {0, 0, 0};
        for (long b = 0; b < n; ++b) {
            if (b == a) continue;
            const double* vb = v + 3 * b;
            const double* Ab = an + 3 * b;
            double d[3] = {x[3 * b] - x[3 * a], x[3 * b + 1] - x[3 * a + 1], x[3 * b + 2] - x[3 * a + 2]};
            double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (d2 == 0.0) continue;
            double inv = 1.0 / sqrt(d2 + eps2);
            double nab[3] = {-d[0] * inv, -d[1] * inv, -d[2] * inv};
            double vb2 = vb[0] * vb[0] + vb[1] * vb[1] + vb[2] * vb[2];
            double vab = va[0] * vb[0] + va[1] * vb[1] + va[2] * vb[2];
            double nvb = nab[0] * vb[0] + nab[1] * vb[1] + nab[2] * vb[2];
            double nva = nab[0] * va[0] + nab[1] * va[1] + nab[2] * va[2];
            double dA = d[0] * Ab[0] + d[1] * Ab[1] + d[2] * Ab[2];
            double br = -4.0 * phi[a] - phi[b] + va2 + 2.0 * vb2 - 4.0 * vab - 1.5 * nvb * nvb + 0.5 * dA;
            double f = G * m[b] * inv * inv;
            double w = 4.0 * nva - 3.0 * nvb;
            double g7 = 3.5 * G * m[b] * inv;
            for (int k = 0; k < 3; ++k) pn[k] += f * (-nab[k] * br + w * (va[k] - vb[k])) + g7 * Ab[k];
        }
        for (int k = 0; k < 3; ++k) acc[3 * a + k] = an[3 * a + k] + inv_c2 * pn[k];
    }
}

/* The EIH accelerations of one system (exported for the tests). */
void orc_eih_acc(long n, const double* x, const double* v, const double* m, double G, double inv_c, double eps2,
                 double* acc) {
    ens_eih_acc(n, x, v, m, G, inv_c * inv_c, eps2, acc);
}

typedef struct {
    const int64_t* off; double *pos, *vel; const double* m; double G, inv_c, eps2, dt; int pn, integrator;
    long nsteps;
} ens_ctx;

static void ens_range(void* c_, long lo, long hi) {
    ens_ctx* c = (ens_ctx*)c_;
    double cc[4], dd[3];
    int ns;
    orc_ens_coeffs(c->integrator, cc, dd, &ns);
    double acc[64 * 3], a[3];
    for (long s = lo; s < hi; ++s) {
        long b0 = c->off[s], n = c->off[s + 1] - b0;
        double* x = c->pos + 3 * b0;
        double* v = c->vel + 3 * b0;
        const double* m = c->m + b0;
        for (long step = 0; step < c->nsteps; ++step) {
            for (int st = 0; st < ns; ++st) {
                for (long i = 0; i < 3 * n; ++i) x[i] += cc[st] * c->dt * v[i];
                if ((c->pn & EIH_FLAG) && (c->pn & PN1_FLAG)) {
                    ens_eih_acc(n, x, v, m, c->G, c->inv_c * c->inv_c, c->eps2, acc);
                } else {
                    for (long i = 0; i < n; ++i) {
                        double ax = 0, ay = 0, az = 0;
                        for (long j = 0; j < n; ++j) {
                            if (j == i) continue;
                            orc_pair_acc(c->G, c->inv_c, c->eps2, c->pn, m[i], m[j], v + 3 * i, v + 3 * j,
                                         x + 3 * i, x + 3 * j, a);
                            ax += a[0]; ay += a[1]; az += a[2];
                        }
                        acc[3 * i] = ax; acc[3 * i + 1] = ay; acc[3 * i + 2] = az;
                    }
                }
                for (long i = 0; i < 3 * n; ++i) v[i] += dd[st] * c->dt * acc[i];
            }
            for (long i = 0; i < 3 * n; ++i) x[i] += cc[ns] * c->dt * v[i];
        }
    }
}

/* Advances every system (bodies off[s]..off[s+1]-1, at most 64) nsteps. */
void orc_ens_run(long nsys, const int64_t* off, double* pos, double* vel, const double* m, double G, double inv_c,
                 double eps2, int pn, int integrator, double dt, long nsteps) {
    ens_ctx c = {off, pos, vel, m, G, inv_c, eps2, dt, pn, integrator, nsteps};
    orc_parallel(nsys, ens_range, &c);
}

/* Per-system energy: Newtonian (Plummer-softened potential) plus, with the
 * PN1 bit, the two-body 1PN energy summed over pairs (harmonic gauge,
 * r = sqrt(d.d + eps2), n = d/r):
 *   (1/c^2) [ sum_i 3/8 m_i v_i^4
 *           + sum_{i<j} G m_i m_j/(2r) (3(v_i^2 + v_j^2) - 7 v_i.v_j - (n.v_i)(n.v_j))
 *           + sum_{i<j} G^2 m_i m_j (m_i + m_j)/(2 r^2) ]
 * (the energy of the two-body Einstein-Infeld-Hoffmann Lagrangian, whose
 * equations of motion are the pairwise 1PN law). With the EIH bit the last
 * sum is the N-body one, (1/2) sum_a m_a phi_a^2 with phi_a = sum_{b != a}
 * G m_b / r_ab (the pair sum above plus the three-body terms
 * (1/2) sum_a sum_{b != a} sum_{c != a, b} G^2 m_a m_b m_c / (r_ab r_ac)): the
 * conserved energy of the N-body EIH Lagrangian. The kicks evaluate the
 * velocity-dependent force at the current velocity, as the reference's
 * integrators do, so the PN part is integrated to first order in dt. */
void orc_ens_energy(long nsys, const int64_t* off, const double* pos, const double* vel, const double* m,
                    double G, double inv_c, double eps2, int pn, double* e_out) {
    for (long s = 0; s < nsys; ++s) {
        long b0 = off[s], n = off[s + 1] - b0;
        const double* x = pos + 3 * b0;
        const double* v = vel + 3 * b0;
        const double* mm = m + b0;
        double e = 0, e1 = 0;
        const int eih = (pn & EIH_FLAG) != 0;
        for (long i = 0; i < n; ++i) {
            double v2 = v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2];
            e += 0.5 * mm[i] * v2;
            e1 += 0.375 * mm[i] * v2 * v2;
            if (eih) {
                double phi = 0;
                for (long j = 0; j < n; ++j) {
                    if (j == i) continue;
                    double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
                    double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                    if (d2 > 0.0) phi += G * mm[j] / sqrt(d2 + eps2);
                }
                e1 += 0.5 * mm[i] * phi * phi;
            }
            for (long j = i + 1; j < n; ++j) {
                double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
                double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2);
                e -= G * mm[i] * mm[j] / r;
                double vj2 = v[3 * j] * v[3 * j] + v[3 * j + 1] * v[3 * j + 1] + v[3 * j + 2] * v[3 * j + 2];
                double vij = v[3 * i] * v[3 * j] + v[3 * i + 1] * v[3 * j + 1] + v[3 * i + 2] * v[3 * j + 2];
                double nvi = (d[0] * v[3 * i] + d[1] * v[3 * i + 1] + d[2] * v[3 * i + 2]) / r;
                double nvj = (d[0] * v[3 * j] + d[1] * v[3 * j + 1] + d[2] * v[3 * j + 2]) / r;
                e1 += G * mm[i] * mm[j] / (2.0 * r) * (3.0 * (v2 + vj2) - 7.0 * vij - nvi * nvj);
                if (!eih) e1 += G * G * mm[i] * mm[j] * (mm[i] + mm[j]) / (2.0 * r * r);
            }
        }
        e_out[s] = e + ((pn & PN1_FLAG) ? inv_c * inv_c * e1 : 0.0);
    }
}

/* ------------------------------------------------------------------------ */
/* adjoint of the KDK leapfrog (FP64 reverse mode, no checkpointing)         */
/* ------------------------------------------------------------------------ */
/* Forward (h = dt/2, A = Newtonian softened acceleration, orc_kdk's map):
 *   v' = v_n + h A(x_n);  x_{n+1} = x_n + dt v';  v_{n+1} = v' + h A(x_{n+1})
 * Loss L = (1/N) sum_i |x_T,i - x*_i|^2. Reverse sweep, lx = dL/dx, lv = dL/dv:
 *   seed lx = (2/N)(x_T - x*), lv = 0, lm = 0
 *   for n = T-1 .. 0:  lv' = lv + dt lx;  w = c_n h lv'  (c_n = 2 for n >= 1,
 *                      1 for n = 0: A(x_n) enters the closing kick of step n-1
 *                      and the opening kick of step n with the same cotangent)
 *                      lx += J(x_n)^T w;  lm += (dA/dm)^T w;  lv = lv'
 * with d = x_j - x_k, s = (d.d + eps2)^(-1/2):
 *   (J^T w)_k  = G sum_{j != k} [ s^3 u - 3 s^5 d (d.u) ],  u = m_k w_j - m_j w_k
 *   (dA/dm)^T w at k = -G sum_{j != k} s^3 (w_j . d)
 * The reference has no adjoint; this is the FP64 CPU reverse-mode reference. */
void orc_adjoint_pair(long n, const double* x, const double* m, const double* w, double G, double eps2,
                      double* jt, double* gm) {
    for (long k = 0; k < n; ++k) {
        double jx = 0, jy = 0, jz = 0, g = 0;
        for (long j = 0; j < n; ++j) {
            if (j == k) continue;
            double d[3] = {x[3 * j] - x[3 * k], x[3 * j + 1] - x[3 * k + 1], x[3 * j + 2] - x[3 * k + 2]};
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
            double s = 1.0 / sqrt(r2);
            double s3 = s * s * s, s5 = s3 * s * s;
            double u[3] = {m[k] * w[3 * j] - m[j] * w[3 * k], m[k] * w[3 * j + 1] - m[j] * w[3 * k + 1],
                           m[k] * w[3 * j + 2] - m[j] * w[3 * k + 2]};
            double du = d[0] * u[0] + d[1] * u[1] + d[2] * u[2];
            jx += s3 * u[0] - 3.0 * s5 * d[0] * du;
            jy += s3 * u[1] - 3.0 * s5 * d[1] * du;
            jz += s3 * u[2] - 3.0 * s5 * d[2] * du;
            g -= s3 * (w[3 * j] * d[0] + w[3 * j + 1] * d[1] + w[3 * j + 2] * d[2]);
        }
        jt[3 * k] = G * jx; jt[3 * k + 1] = G * jy; jt[3 * k + 2] = G * jz;
        gm[k] = G * g;
    }
}

/* Loss and gradients dL/dx0, dL/dv0, dL/dm of the trajectory from (x0, v0, m).
 * Keeps every position of the trajectory (small n and T only). */
double orc_adjoint(long n, const double* x0, const double* v0, const double* m, const double* target, double G,
                   double eps2, double dt, long T, double* gx, double* gv, double* gmass) {
    double* xs = (double*)malloc((size_t)(T + 1) * n * 3 * sizeof(double));
    double* v = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* a = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* w = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* jt = (double*)malloc((size_t)n * 3 * sizeof(double));
    double* gm = (double*)malloc((size_t)n * sizeof(double));
    const double h = 0.5 * dt;
    memcpy(xs, x0, (size_t)n * 3 * sizeof(double));
    memcpy(v, v0, (size_t)n * 3 * sizeof(double));
    orc_allpairs(n, xs, NULL, m, G, 0.0, eps2, 1, 0, NULL, a);
    for (long t = 0; t < T; ++t) {
        double* xc = xs + (size_t)t * n * 3;
        double* xn = xs + (size_t)(t + 1) * n * 3;
        for (long i = 0; i < 3 * n; ++i) { v[i] += h * a[i]; xn[i] = xc[i] + dt * v[i]; }
        orc_allpairs(n, xn, NULL, m, G, 0.0, eps2, 1, 0, NULL, a);
        for (long i = 0; i < 3 * n; ++i) v[i] += h * a[i];
    }
    const double* xT = xs + (size_t)T * n * 3;
    double loss = 0.0;
    for (long i = 0; i < 3 * n; ++i) {
        double d = xT[i] - target[i];
        loss += d * d;
        gx[i] = 2.0 * d / (double)n;
        gv[i] = 0.0;
    }
    loss /= (double)n;
    for (long k = 0; k < n; ++k) gmass[k] = 0.0;
    for (long t = T - 1; t >= 0; --t) {
        const double c = t >= 1 ? 2.0 : 1.0;
        for (long i = 0; i < 3 * n; ++i) { gv[i] += dt * gx[i]; w[i] = c * h * gv[i]; }
        orc_adjoint_pair(n, xs + (size_t)t * n * 3, m, w, G, eps2, jt, gm);
        for (long i = 0; i < 3 * n; ++i) gx[i] += jt[i];
        for (long k = 0; k < n; ++k) gmass[k] += gm[k];
    }
    free(xs); free(v); free(a); free(w); free(jt); free(gm);
    return loss;
}

/* acc and body_count (optional) are indexed by body (input order). */
void orc_lbvh_forces(long n, int group, const int32_t* left, const int32_t* right, const int32_t* parent,
                     const int32_t* rlo, const int32_t* rhi, const int32_t* perm,
                     const double* pos, const double* node_mass, const double* node_com,
                     const float* rcrit2, double G, double eps2, double* acc, int32_t* body_count) {
    if (group <= 0) group = ORC_GROUP;
    int32_t* gs = (int32_t*)malloc((size_t)n * 4);
    int32_t* gc = (int32_t*)malloc((size_t)n * 4);
    long ng = orc_groups(n, group, parent, rlo, rhi, gs, gc);
    trav_ctx c = {n, gs, gc, left, right, perm, pos, node_mass, node_com, rcrit2, G, eps2, acc, body_count,
                  NULL, NULL, 0.0, 0};
    orc_parallel(ng, trav_range, &c);
    free(gs);
    free(gc);
}

/* Node velocities in NodesArray::unite form (barnes_hut.cpp:150): leaf k =
 * vel[perm[k]]; internal v = (v_R m_R + v_L m_L) / M with M = node_mass[v]
 * (from orc_bottom_up), or (v_R + v_L) / 2 when M <= 0. Post-order. */
void orc_node_velocities(long n, const int32_t* left, const int32_t* right, const int32_t* perm,
                         const double* vel, const double* node_mass, double* node_vel) {
    for (long k = 0; k < n; ++k)
        for (int a = 0; a < 3; ++a) node_vel[3 * k + a] = vel[3 * (long)perm[k] + a];
    if (n < 2) return;
    long total = 2 * n - 1;
    int32_t* stack = (int32_t*)malloc((size_t)total * 4);
    char* done = (char*)calloc((size_t)total, 1);
    long sp = 0;
    stack[sp++] = (int32_t)n;
    while (sp > 0) {
        int32_t v = stack[sp - 1];
        int32_t L = left[v], R = right[v];
        if (v >= n && (!done[L] && L >= n)) { stack[sp++] = L; continue; }
        if (v >= n && (!done[R] && R >= n)) { stack[sp++] = R; continue; }
        sp--;
        if (v < n) { done[v] = 1; continue; }
        double M = node_mass[v];
        for (int a = 0; a < 3; ++a)
            node_vel[3 * v + a] = M > 0.0
                ? (node_vel[3 * R + a] * node_mass[R] + node_vel[3 * L + a] * node_mass[L]) / M
                : 0.5 * (node_vel[3 * R + a] + node_vel[3 * L + a]);
        done[v] = 1;
    }
    free(stack);
    free(done);
}

/* The group walk with a post-Newtonian force law: the same lists as
 * orc_lbvh_forces, each entry through orc_pair_acc with the target's velocity
 * and the node's (node_vel from orc_node_velocities). */
void orc_lbvh_forces_pn(long n, int group, const int32_t* left, const int32_t* right, const int32_t* parent,
                        const int32_t* rlo, const int32_t* rhi, const int32_t* perm,
                        const double* pos, const double* vel, const double* node_mass, const double* node_com,
                        const double* node_vel, const float* rcrit2, double G, double inv_c, double eps2, int pn,
                        double* acc, int32_t* body_count) {
    if (group <= 0) group = ORC_GROUP;
    int32_t* gs = (int32_t*)malloc((size_t)n * 4);
    int32_t* gc = (int32_t*)malloc((size_t)n * 4);
    long ng = orc_groups(n, group, parent, rlo, rhi, gs, gc);
    trav_ctx c = {n, gs, gc, left, right, perm, pos, node_mass, node_com, rcrit2, G, eps2, acc, body_count,
                  vel, node_vel, inv_c, pn};
    orc_parallel(ng, trav_range, &c);
    free(gs);
    free(gc);
}
