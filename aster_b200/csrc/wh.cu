// Wisdom-Holman planetary integrator on the device: body 0 is the central
// mass, the others (planets, and test particles of zero mass) move on Kepler
// orbits about it, perturbed by one another.
//
// Replaces update_WH_planetary (src/physics/tool_chain_impl.cpp:186-290) and
// its OpenCL form (include/Aster/kernels/WH_planetary.cl.h, src/utils/
// updater.cpp:90-122). Those kick every body with the solver's full
// acceleration, the central body's pull included, after a Kepler drift that
// has already integrated that pull: a circular orbit falls to a third of its
// radius within one period. This is the published method they aim at, in
// democratic heliocentric coordinates (Wisdom & Holman 1991; Duncan, Levison &
// Lee 1998): Q_i = x_i - x_0, V_i = v_i - v_cm (i >= 1),
//   A  Kepler:       V_i^2/2 - G m_0/|Q_i|           (per body, exact)
//   B  interaction:  -G m_i m_j / |Q_i - Q_j|, i, j >= 1 (kick)
//   C  linear drift: |sum_i m_i V_i|^2 / (2 m_0)     (Q_i += P/m_0 h)
// one step = C(h) B(h) A(dt) C(h) B(h), h = dt/2. B and C commute, so the
// interaction at a step's end serves the next step's first kick: one force
// evaluation per step. The interaction is the all-pairs kernel on the working
// state with the central body's mass set to zero (it then acts on nobody),
// its closing kick applying B. The barycentre moves uniformly; the inertial
// state is rebuilt at the end of the call.
//
// Kepler drift: universal variables (Stumpff functions c2, c3), the
// Laguerre-Conway iteration on the universal Kepler equation from
// chi = sqrt(mu) dt / r, then the f and g functions; at most 64 iterations,
// after which the body is left as it was and ASTER_ERR_KEPLER is reported.
#include <algorithm>

#include "aster_internal.cuh"

namespace {

constexpr int WH_BLOCK = 256;

// state scalars in ctx->wh after the partials: [0] m0, [1] M, [2..4] x_cm,
// [5..7] v_cm, [8..11] reduction result (sum m a.x, .y, .z, sum m), [12..14]
// sum m v, [16..18] sum m Q, [20..22] sum m x, [24..27] the second slot for P
// (k_wh_cba reads P from one slot and writes the next P to the other), [30] the
// reductions' block counter (an unsigned int, zero between launches)
struct WhLayout {
    int64_t nb;  // reduction blocks
    double* part;
    double* st;
};

WhLayout wh_layout(aster_ctx* c) {
    WhLayout L;
    L.nb = std::min<int64_t>((c->n + WH_BLOCK - 1) / WH_BLOCK, (int64_t)c->sm_count * 4);
    if (L.nb < 1) L.nb = 1;
    L.part = c->wh.as<double>();
    L.st = L.part + 4 * L.nb;
    return L;
}

// Block-wide sum of each thread's s[0..3] into part[4 * block]; the last block
// to finish then adds the partials in block order (deterministic whichever
// block is last), writes the total to out4[0..3] and re-arms *done (zero
// between launches). Every thread of every block calls it once.
__device__ __forceinline__ void block_sum4_last(const double s[4], double* part, unsigned int* done,
                                                double* out4) {
    __shared__ double red[4][WH_BLOCK / 4];
    __shared__ bool last;
    for (int k = 0; k < 4; ++k) {
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0;
        for (int w = 0; w < WH_BLOCK / 32; ++w) v += red[threadIdx.x][w];
        part[blockIdx.x * 4 + threadIdx.x] = v;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // thread t adds component t & 3 of blocks g, g + G, g + 2G, ... (g = t >> 2,
    // G = WH_BLOCK / 4), then thread k < 4 adds the G group sums in order
    const int k = threadIdx.x & 3, g = threadIdx.x >> 2;
    double v = 0;
    for (unsigned b = g; b < gridDim.x; b += WH_BLOCK / 4) v += __ldcg(part + 4 * b + k);
    red[k][g] = v;
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0;
        for (int q = 0; q < WH_BLOCK / 4; ++q) t += red[threadIdx.x][q];
        out4[threadIdx.x] = t;
    }
    if (threadIdx.x == 0) *done = 0u;
}

// sum over i in [i0, n) of (m_i a_i, m_i), m from pm[i].w, into out4[0..3]
__global__ void __launch_bounds__(WH_BLOCK) k_wh_reduce(int64_t n, int64_t i0, const double4* __restrict__ pm,
                                                        const double4* __restrict__ a, double* part,
                                                        unsigned int* done, double* out4) {
    double s[4] = {0, 0, 0, 0};
    for (int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double m = pm[i].w;
        const double4 x = a[i];
        s[0] += m * x.x; s[1] += m * x.y; s[2] += m * x.z; s[3] += m;
    }
    block_sum4_last(s, part, done, out4);
}

// inertial -> working state. Reads the reductions: st[8..11] = (sum m x, M)
// over all bodies, the previous launch's copy of (sum m v) in st[12..14].
__global__ void __launch_bounds__(WH_BLOCK) k_wh_to_dhc(int64_t n, double4* __restrict__ pm, double4* __restrict__ vel,
                                                        double* __restrict__ st) {
    const double M = st[11];
    const double vcx = st[12] / M, vcy = st[13] / M, vcz = st[14] / M;
    const double4 x0 = pm[0];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (i == 0) continue;
        double4 p = pm[i], v = vel[i];
        p.x -= x0.x; p.y -= x0.y; p.z -= x0.z;
        v.x -= vcx; v.y -= vcy; v.z -= vcz;
        pm[i] = p;
        vel[i] = v;
    }
}

// Stumpff functions c2(z) = (1 - cos sqrt z) / z, c3(z) = (sqrt z - sin sqrt z) / z^1.5.
// |z| < 0.5: their Maclaurin series c2 = sum (-z)^k / (2k+2)!, c3 = sum (-z)^k /
// (2k+3)!, ten terms (the first omitted term is below 2^-53 of the sum) in
// Horner form with the reciprocal factorials as constants (folded at compile
// time, each correctly rounded).
__device__ __forceinline__ void stumpff(double z, double& c2, double& c3) {
    if (fabs(z) < 0.5) {
        const double x = -z;
        c2 = 1.0 / 2432902008176640000.0;                     // 1/20!
        c2 = fma(c2, x, 1.0 / 6402373705728000.0);            // 1/18!
        c2 = fma(c2, x, 1.0 / 20922789888000.0);              // 1/16!
        c2 = fma(c2, x, 1.0 / 87178291200.0);                 // 1/14!
        c2 = fma(c2, x, 1.0 / 479001600.0);                   // 1/12!
        c2 = fma(c2, x, 1.0 / 3628800.0);                     // 1/10!
        c2 = fma(c2, x, 1.0 / 40320.0);                       // 1/8!
        c2 = fma(c2, x, 1.0 / 720.0);                         // 1/6!
        c2 = fma(c2, x, 1.0 / 24.0);                          // 1/4!
        c2 = fma(c2, x, 0.5);                                 // 1/2!
        c3 = 1.0 / 51090942171709440000.0;                    // 1/21!
        c3 = fma(c3, x, 1.0 / 121645100408832000.0);          // 1/19!
        c3 = fma(c3, x, 1.0 / 355687428096000.0);             // 1/17!
        c3 = fma(c3, x, 1.0 / 1307674368000.0);               // 1/15!
        c3 = fma(c3, x, 1.0 / 6227020800.0);                  // 1/13!
        c3 = fma(c3, x, 1.0 / 39916800.0);                    // 1/11!
        c3 = fma(c3, x, 1.0 / 362880.0);                      // 1/9!
        c3 = fma(c3, x, 1.0 / 5040.0);                        // 1/7!
        c3 = fma(c3, x, 1.0 / 120.0);                         // 1/5!
        c3 = fma(c3, x, 1.0 / 6.0);                           // 1/3!
    } else if (z > 0.0) {
        const double s = sqrt(z), h = sin(0.5 * s);
        c2 = 2.0 * h * h / z;
        c3 = (s - sin(s)) / (z * s);
    } else {
        const double s = sqrt(-z);
        c2 = (cosh(s) - 1.0) / (-z);
        c3 = (sinh(s) - s) / (-z * s);
    }
}

// Advances (r, v) along the Kepler orbit about mu for dt; false (unchanged)
// when r = 0 or the iteration does not converge.
__device__ bool kepler_drift(double3& r, double3& v, double mu, double dt) {
    const double r0 = sqrt(r.x * r.x + r.y * r.y + r.z * r.z);
    if (!(r0 > 0.0)) return false;
    const double v2 = v.x * v.x + v.y * v.y + v.z * v.z;
    const double smu = sqrt(mu);
    const double s0 = (r.x * v.x + r.y * v.y + r.z * v.z) / smu;
    const double a = 2.0 / r0 - v2 / mu;
    const double b = 1.0 - a * r0;
    double chi = smu * dt / r0, c2 = 0.5, c3 = 1.0 / 6.0;
    bool ok = false;
    for (int it = 0; it < 64; ++it) {
        const double z = a * chi * chi;
        stumpff(z, c2, c3);
        const double F = r0 * chi + s0 * chi * chi * c2 + b * chi * chi * chi * c3 - smu * dt;
        const double Fp = r0 + s0 * chi * (1.0 - z * c3) + b * chi * chi * c2;
        const double Fpp = s0 * (1.0 - z * c2) + b * chi * (1.0 - z * c3);
        const double disc = fabs(16.0 * Fp * Fp - 20.0 * F * Fpp);
        const double den = Fp + (Fp >= 0.0 ? 1.0 : -1.0) * sqrt(disc);
        const double d = den != 0.0 ? 5.0 * F / den : F / Fp;
        chi -= d;
        if (fabs(d) <= 1e-15 * (1.0 + fabs(chi))) {
            ok = true;
            break;
        }
    }
    if (!ok || !isfinite(chi)) return false;
    const double z = a * chi * chi;
    stumpff(z, c2, c3);
    const double f = 1.0 - chi * chi * c2 / r0;
    const double g = dt - chi * chi * chi * c3 / smu;
    const double3 rn = make_double3(f * r.x + g * v.x, f * r.y + g * v.y, f * r.z + g * v.z);
    const double rr = sqrt(rn.x * rn.x + rn.y * rn.y + rn.z * rn.z);
    const double fd = smu / (rr * r0) * chi * (z * c3 - 1.0);
    const double gd = 1.0 - chi * chi * c2 / rr;
    v = make_double3(fd * r.x + gd * v.x, fd * r.y + gd * v.y, fd * r.z + gd * v.z);
    r = rn;
    return true;
}

// Per body i >= 1: C(hc) with P = pin[0..2], B(hb) with the cached
// interaction acc, A(dt); then P = sum m_i V_i after the drift into pout[0..2]
// (pout[3] = sum m_i), pin and pout distinct slots of the state scalars.
__global__ void __launch_bounds__(WH_BLOCK) k_wh_cba(int64_t n, double4* __restrict__ pm, double4* __restrict__ vel,
                                                     const double4* __restrict__ acc, const double* st,
                                                     const double* pin, double hc, double hb, double mu, double dt,
                                                     int* __restrict__ err, double* part, unsigned int* done,
                                                     double* pout) {
    const double m0 = st[0];
    const double px = pin[0] / m0 * hc, py = pin[1] / m0 * hc, pz = pin[2] / m0 * hc;
    double sum[4] = {0, 0, 0, 0};
    for (int64_t i = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double4 p = pm[i], v = vel[i];
        const double4 a = acc[i];
        double3 r = make_double3(p.x + px, p.y + py, p.z + pz);
        double3 u = make_double3(v.x + a.x * hb, v.y + a.y * hb, v.z + a.z * hb);
        if (!kepler_drift(r, u, mu, dt)) atomicOr(err, ASTER_DEVERR_KEPLER);
        pm[i] = make_double4(r.x, r.y, r.z, p.w);
        vel[i] = make_double4(u.x, u.y, u.z, v.w);
        sum[0] += p.w * u.x; sum[1] += p.w * u.y; sum[2] += p.w * u.z; sum[3] += p.w;
    }
    block_sum4_last(sum, part, done, pout);
}

// C(h) alone with P = pin[0..2] (a run's last half step; B follows in the
// force launch's closing kick).
__global__ void __launch_bounds__(WH_BLOCK) k_wh_c(int64_t n, double4* __restrict__ pm, const double* st,
                                                   const double* pin, double h) {
    const double m0 = st[0];
    const double px = pin[0] / m0 * h, py = pin[1] / m0 * h, pz = pin[2] / m0 * h;
    for (int64_t i = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double4 p = pm[i];
        p.x += px; p.y += py; p.z += pz;
        pm[i] = p;
    }
}

// working -> inertial state: x_0 = x_cm + v_cm T - S/M, x_i = x_0 + Q_i,
// v_i = v_cm + V_i, v_0 = v_cm - P/m_0; S = st[16..18] (sum m Q), P = st[8..10].
__global__ void __launch_bounds__(WH_BLOCK) k_wh_from_dhc(int64_t n, double4* __restrict__ pm,
                                                          double4* __restrict__ vel, const double* __restrict__ st,
                                                          double T) {
    const double m0 = st[0], M = st[1];
    const double vcx = st[5], vcy = st[6], vcz = st[7];
    const double x0x = st[2] + vcx * T - st[16] / M, x0y = st[3] + vcy * T - st[17] / M,
                 x0z = st[4] + vcz * T - st[18] / M;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (i == 0) {
            pm[0] = make_double4(x0x, x0y, x0z, m0);
            vel[0] = make_double4(vcx - st[8] / m0, vcy - st[9] / m0, vcz - st[10] / m0, 0.0);
            continue;
        }
        double4 p = pm[i], v = vel[i];
        p.x += x0x; p.y += x0y; p.z += x0z;
        v.x += vcx; v.y += vcy; v.z += vcz;
        pm[i] = p;
        vel[i] = v;
    }
}

// st[0..7] = (m0, M, x_cm, v_cm) from the reductions; zeroes the central mass.
__global__ void k_wh_setup(double4* __restrict__ pm, double* __restrict__ st) {
    const double M = st[11];
    st[0] = pm[0].w;
    st[1] = M;
    st[2] = st[20] / M; st[3] = st[21] / M; st[4] = st[22] / M;
    st[5] = st[12] / M; st[6] = st[13] / M; st[7] = st[14] / M;
    pm[0].w = 0.0;  // the central body acts on nobody in the interaction
}

__global__ void k_wh_copy3(double* __restrict__ st, int from, int to) {
    if (threadIdx.x < 4) st[to + threadIdx.x] = st[from + threadIdx.x];
}

}  // namespace

// ASTER_OK, or the error of the last launch
static int wh_launch_status() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ASTER_OK : aster_cuda_fail(e, "WH kernel launch", __FILE__, __LINE__);
}

// sum over i in [i0, n) of (m_i a_i, m_i) into st[8..11]
static int wh_reduce(aster_ctx* c, const WhLayout& L, int64_t i0, const double4* a) {
    k_wh_reduce<<<(unsigned)L.nb, WH_BLOCK, 0, c->stream>>>(c->n, i0, c->pm.as<double4>(), a, L.part,
                                                           reinterpret_cast<unsigned int*>(L.st + 30), L.st + 8);
    ASTER_CUDA(cudaGetLastError());
    c->stats.kernels += 1;
    return ASTER_OK;
}

static int wh_check(aster_ctx* c, const aster_params* p, int precision, int nsteps) {
    if (!c || nsteps < 0) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    if (c->n < 2) return ASTER_ERR_INVALID_ARG;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    if (p->force_law & ~ASTER_NEWTON) return ASTER_ERR_UNSUPPORTED;
    if (!(p->G > 0.0)) return ASTER_ERR_INVALID_ARG;
    return ASTER_OK;
}

// The central body's mass (synchronises the stream): must be positive.
int aster_wh_central_mass(aster_ctx* c, double* m0) {
    double4 b0;
    ASTER_CUDA(cudaMemcpyAsync(&b0, c->pm.ptr, sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
    ASTER_CUDA(cudaStreamSynchronize(c->stream));
    *m0 = b0.w;
    return b0.w > 0.0 ? ASTER_OK : ASTER_ERR_INVALID_ARG;
}

// Enqueues nsteps Wisdom-Holman steps (no synchronisation); m0 = the central
// mass (> 0, from aster_wh_central_mass). The state is inertial before and after.
int aster_wh_enqueue(aster_ctx* c, const aster_params* p, int precision, int nsteps, double m0) {
    ASTER_TRY(wh_check(c, p, precision, nsteps));
    const int64_t n = c->n;
    const int64_t nbmax = std::min<int64_t>((n + WH_BLOCK - 1) / WH_BLOCK, (int64_t)c->sm_count * 4);
    ASTER_TRY(c->wh.ensure((size_t)(4 * std::max<int64_t>(nbmax, 1) + 32) * sizeof(double)));
    const WhLayout L = wh_layout(c);
    ASTER_CUDA(cudaMemsetAsync(L.st + 30, 0, sizeof(double), c->stream));  // arm the reduction counter
    c->mixed_valid = false;  // the steps move positions and velocities (mixed runs refresh as they go)
    const double mu = p->G * m0;
    double4* pm = c->pm.as<double4>();
    double4* vel = c->vel.as<double4>();
    const int grid = (int)L.nb;
    const double dt = p->dt, h = 0.5 * dt;
    // barycentre: (sum m x, M) -> st[20..22], st[11]; (sum m v) -> st[12..14]
    ASTER_TRY(wh_reduce(c, L, 0, pm));
    k_wh_copy3<<<1, 32, 0, c->stream>>>(L.st, 8, 20);
    ASTER_TRY(wh_reduce(c, L, 0, vel));
    k_wh_copy3<<<1, 32, 0, c->stream>>>(L.st, 8, 12);
    k_wh_setup<<<1, 1, 0, c->stream>>>(pm, L.st);
    k_wh_to_dhc<<<grid, WH_BLOCK, 0, c->stream>>>(n, pm, vel, L.st);
    ASTER_CUDA(cudaGetLastError());
    c->stats.kernels += 4;
    int st = ASTER_OK;
    int done = 0;  // Kepler drifts taken: the barycentre advances by done * dt
    // Steps C(h) B(h) A(dt) C(h) B(h) in sequence: between two drifts A the
    // C(h) B(h) C(h) B(h) collapse to C(dt) B(dt) (B leaves P = sum m V
    // unchanged, and the interaction does not change under the uniform shift
    // C), so a run is C(h) B(h) A [C(dt) B(dt) A] x (nsteps - 1) C(h) B(h):
    // one interaction launch and one k_wh_cba (with P for the next C) a step.
    unsigned int* cnt = reinterpret_cast<unsigned int*>(L.st + 30);
    double* pslot[2] = {L.st + 8, L.st + 24};
    int cur = 0;
    for (int s = 0; s < nsteps && st == ASTER_OK; ++s) {
        if (precision == ASTER_MIXED && (st = aster_refresh_mixed(c)) != ASTER_OK) break;
        if ((st = aster_allpairs_launch(c, p, precision, false, n, nullptr, nullptr)) != ASTER_OK) break;
        if (s == 0 && (st = wh_reduce(c, L, 1, vel)) != ASTER_OK) break;  // P of the initial state
        const double hcb = s == 0 ? h : dt;
        k_wh_cba<<<grid, WH_BLOCK, 0, c->stream>>>(n, pm, vel, c->acc.as<double4>(), L.st, pslot[cur], hcb, hcb, mu,
                                                   dt, c->err_dev, L.part, cnt, pslot[cur ^ 1]);
        if ((st = wh_launch_status()) != ASTER_OK) break;
        cur ^= 1;
        ++done;
        c->stats.kernels += 1;
    }
    if (st == ASTER_OK && done > 0) {  // the last C(h) B(h)
        k_wh_c<<<grid, WH_BLOCK, 0, c->stream>>>(n, pm, L.st, pslot[cur], h);
        st = wh_launch_status();
        c->stats.kernels += 1;
        if (st == ASTER_OK && precision == ASTER_MIXED) st = aster_refresh_mixed(c);
        if (st == ASTER_OK) st = aster_allpairs_launch(c, p, precision, true, n, nullptr, nullptr);  // + B(h)
    }
    // back to the inertial state (also after an error, so the state stays meaningful)
    if (wh_reduce(c, L, 1, pm) == ASTER_OK) {  // S = sum m Q
        k_wh_copy3<<<1, 32, 0, c->stream>>>(L.st, 8, 16);
        if (wh_reduce(c, L, 1, vel) == ASTER_OK) {  // P
            k_wh_from_dhc<<<grid, WH_BLOCK, 0, c->stream>>>(n, pm, vel, L.st, dt * done);
            c->stats.kernels += 2;
        }
    }
    c->acc_valid = false;  // acc holds the interaction, not the full acceleration
    if (precision == ASTER_MIXED && st == ASTER_OK) st = aster_refresh_mixed(c);
    return st;
}

extern "C" int aster_wh_steps(aster_ctx* c, const aster_params* p, int precision, int nsteps) {
    ASTER_TRY(wh_check(c, p, precision, nsteps));
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    double m0 = 0.0;
    ASTER_TRY(aster_wh_central_mass(c, &m0));
    cudaEventRecord(c->ev[0], c->stream);
    int st = aster_wh_enqueue(c, p, precision, nsteps, m0);
    cudaEventRecord(c->ev[1], c->stream);
    const int fin = aster_finish(c);
    if (st == ASTER_OK) st = fin;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    return st;
}
