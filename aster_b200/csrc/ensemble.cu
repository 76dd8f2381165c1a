// Batched ensembles of few-body systems: one persistent, graph-captured
// launch integrates thousands of independent systems for many steps.
//
// The reference has no batched solver (a Simulation per system would also
// share Parallelized's function-static pointer, builder_endpoint.cpp:731). The
// pair law is the reference's compute_gravitational
// (src/physics/tool_chain_impl.cpp:120-137) with the pairwise post-Newtonian
// terms of get_pn1 (c^-2, :110-118), get_pn2 (c^-4, :79-107) and get_pn25
// (c^-5, :65-77), selected by the force-law bits; the integrators are
// drift-kick-drift compositions: leapfrog (the map of update_leapfrog,
// tool_chain_impl.cpp:169-185) and Yoshida's (1990) fourth-order triple jump.
//
// Force laws: Newton; Newton + the pairwise post-Newtonian terms (PN level
// 1: 1PN only, 2: any of 1PN/2PN/2.5PN); or (level 3, force-law bit
// ASTER_EIH with ASTER_PN1) the N-body Einstein-Infeld-Hoffmann 1PN
// acceleration, which adds the three-body couplings that get_pn1 leaves out
// (Einstein, Infeld & Hoffmann 1938; Will 1993, sec. 6.2). With
// r_ab = sqrt(|x_a - x_b|^2 + eps2), d = x_b - x_a, n_ab = -d / r_ab,
// Phi_a = sum_{c != a} G m_c / r_ac and A_b the Newtonian acceleration of b:
//   a_a = A_a + c^-2 G sum_{b != a} { m_b / r_ab^2 [d/r_ab B_ab + W_ab (v_a - v_b)] + 7/2 m_b A_b / r_ab }
//   B_ab = -4 Phi_a - Phi_b + v_a^2 + 2 v_b^2 - 4 v_a.v_b - 3/2 (n_ab.v_b)^2 + 1/2 d.A_b
//   W_ab = n_ab.(4 v_a - 3 v_b)
// Level 3 evaluates it in two passes over the system: the first sums A and
// Phi of every body and publishes them beside the positions, the second
// sums the bracketed terms. For two unsoftened bodies it equals get_pn1.
//
// Mapping: one warp per system (at most 64 bodies: one body per lane, or two
// when the system has more than 32), the whole state in registers for the
// entire run; per force evaluation every lane publishes its bodies to the
// warp's shared-memory slab and sums over the slab. Systems are taken largest
// first from a global work counter (longest-processing-time order), so the
// uneven sizes balance across warps. The kernel polls a host-written cancel
// flag every check_every steps; it never waits on anything.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "aster_internal.cuh"
#include "pn.cuh"

namespace {

template <class T>
struct T3 {
    T x, y, z;
};

// Per-body (A, Phi) of EIH pass 1 (level 3), in shared memory after the slabs.
template <bool MIXED>
struct EnsAux;
template <>
struct EnsAux<true> {
    using T = float;
    using T4 = float4;
};
template <>
struct EnsAux<false> {
    using T = double;
    using T4 = double4;
};

struct Coeffs {
    double cdt[4];  // drift coefficients x dt
    double ddt[3];  // kick coefficients x dt
    int nst;        // kicks per step
};

Coeffs make_coeffs(int integrator, double dt) {
    Coeffs k{};
    if (integrator == ASTER_INTEGRATOR_YOSHIDA4) {
        const double cb = std::cbrt(2.0);
        const double w1 = 1.0 / (2.0 - cb), w0 = -cb / (2.0 - cb);
        const double c[4] = {0.5 * w1, 0.5 * (w0 + w1), 0.5 * (w0 + w1), 0.5 * w1};
        const double d[3] = {w1, w0, w1};
        for (int i = 0; i < 4; ++i) k.cdt[i] = c[i] * dt;
        for (int i = 0; i < 3; ++i) k.ddt[i] = d[i] * dt;
        k.nst = 3;
    } else {
        k.cdt[0] = k.cdt[1] = 0.5 * dt;
        k.ddt[0] = dt;
        k.nst = 1;
    }
    return k;
}

template <bool MIXED>
struct EnsSlab;
template <>
struct EnsSlab<true> {
    float4 hi[64];  // (x_hi, y_hi, z_hi, m)
    float4 lo[64];  // (x_lo, y_lo, z_lo, 0)
    float4 v[64];   // (vx, vy, vz, |v|^2)
};
template <>
struct EnsSlab<false> {
    double4 x[64];  // (x, y, z, m)
    double4 v[64];  // (vx, vy, vz, |v|^2)
};

// Sums over j = j0, j0 + js, ... < n (js > 1: the lanes that share a target
// split its sources).
template <int PNL, int UNROLL>
__device__ __forceinline__ void accel_f32(const EnsSlab<true>& s, int n, int j0, int js, float4 hi, float4 lo,
                                          float4 vi, float eps2, float G, const PnK<float>& k, float3& aN, float3& a1,
                                          float3& a2) {
    float ax = 0.f, ay = 0.f, az = 0.f, px = 0.f, py = 0.f, pz = 0.f, qx = 0.f, qy = 0.f, qz = 0.f;
#pragma unroll UNROLL
    for (int j = j0; j < n; j += js) {
        const float4 h = s.hi[j], l = s.lo[j];
        const float dx = (h.x - hi.x) + (l.x - lo.x);
        const float dy = (h.y - hi.y) + (l.y - lo.y);
        const float dz = (h.z - hi.z) + (l.z - lo.z);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
        float inv = rsqrt_approx(r2);
        inv = r2 > 0.f ? inv : 0.f;
        const float inv2 = inv * inv;
        const float sN = h.w * inv * inv2;
        ax = fmaf(dx, sN, ax); ay = fmaf(dy, sN, ay); az = fmaf(dz, sN, az);
        if (PNL > 0) {
            const float4 vj = s.v[j];
            PnPair<float> q;
            q.nx = -dx * inv; q.ny = -dy * inv; q.nz = -dz * inv;
            q.dvx = vi.x - vj.x; q.dvy = vi.y - vj.y; q.dvz = vi.z - vj.z;
            q.inv = inv; q.inv2 = inv2; q.mi = hi.w; q.mj = h.w; q.vi2 = vi.w; q.vj2 = vj.w;
            q.v12 = vi.x * vj.x + vi.y * vj.y + vi.z * vj.z;
            q.nv1 = q.nx * vi.x + q.ny * vi.y + q.nz * vi.z;
            q.nv2 = q.nx * vj.x + q.ny * vj.y + q.nz * vj.z;
            q.G = G;
            pn_terms<PNL>(k, q, px, py, pz, qx, qy, qz);
        }
    }
    aN = make_float3(ax, ay, az);
    a1 = make_float3(px, py, pz);
    a2 = make_float3(qx, qy, qz);
}

template <int PNL, int UNROLL>
__device__ __forceinline__ void accel_f64(const EnsSlab<false>& s, int n, int j0, int js, double4 xi, double4 vi,
                                          double eps2, double G, const PnK<double>& k, double& ax, double& ay,
                                          double& az) {
    double px = 0.0, py = 0.0, pz = 0.0, qx = 0.0, qy = 0.0, qz = 0.0;
    ax = ay = az = 0.0;
#pragma unroll UNROLL
    for (int j = j0; j < n; j += js) {
        const double4 xj = s.x[j];
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
        double inv = r2 > 0.0 ? rsqrt(r2) : 0.0;
        const double inv2 = inv * inv;
        const double sN = xj.w * inv * inv2;
        ax = fma(dx, sN, ax); ay = fma(dy, sN, ay); az = fma(dz, sN, az);
        if (PNL > 0) {
            const double4 vj = s.v[j];
            PnPair<double> q;
            q.nx = -dx * inv; q.ny = -dy * inv; q.nz = -dz * inv;
            q.dvx = vi.x - vj.x; q.dvy = vi.y - vj.y; q.dvz = vi.z - vj.z;
            q.inv = inv; q.inv2 = inv2; q.mi = xi.w; q.mj = xj.w; q.vi2 = vi.w; q.vj2 = vj.w;
            q.v12 = vi.x * vj.x + vi.y * vj.y + vi.z * vj.z;
            q.nv1 = q.nx * vi.x + q.ny * vi.y + q.nz * vi.z;
            q.nv2 = q.nx * vj.x + q.ny * vj.y + q.nz * vj.z;
            q.G = G;
            pn_terms<PNL>(k, q, px, py, pz, qx, qy, qz);
        }
    }
    ax += px + qx; ay += py + qy; az += pz + qz;
}

// EIH pass 1 (level 3): Newtonian sum m_j d / r^3 and potential sum m_j / r
// over j = j0, j0 + js, ... < n (both without G).
template <int UNROLL>
__device__ __forceinline__ void newton_phi_f32(const EnsSlab<true>& s, int n, int j0, int js, float4 hi, float4 lo,
                                               float eps2, float3& aN, float& phi) {
    float ax = 0.f, ay = 0.f, az = 0.f, ph = 0.f;
#pragma unroll UNROLL
    for (int j = j0; j < n; j += js) {
        const float4 h = s.hi[j], l = s.lo[j];
        const float dx = (h.x - hi.x) + (l.x - lo.x);
        const float dy = (h.y - hi.y) + (l.y - lo.y);
        const float dz = (h.z - hi.z) + (l.z - lo.z);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
        float inv = rsqrt_approx(r2);
        inv = r2 > 0.f ? inv : 0.f;
        const float mi = h.w * inv;
        const float sN = mi * inv * inv;
        ax = fmaf(dx, sN, ax); ay = fmaf(dy, sN, ay); az = fmaf(dz, sN, az);
        ph += mi;
    }
    aN = make_float3(ax, ay, az);
    phi = ph;
}

template <int UNROLL>
__device__ __forceinline__ void newton_phi_f64(const EnsSlab<false>& s, int n, int j0, int js, double4 xi,
                                               double eps2, double3& aN, double& phi) {
    double ax = 0.0, ay = 0.0, az = 0.0, ph = 0.0;
#pragma unroll UNROLL
    for (int j = j0; j < n; j += js) {
        const double4 xj = s.x[j];
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
        const double inv = r2 > 0.0 ? rsqrt(r2) : 0.0;
        const double mi = xj.w * inv;
        const double sN = mi * inv * inv;
        ax = fma(dx, sN, ax); ay = fma(dy, sN, ay); az = fma(dz, sN, az);
        ph += mi;
    }
    aN = make_double3(ax, ay, az);
    phi = ph;
}

// EIH pass 2 (level 3): sum over j of m_j / r^2 [d/r B + W (v_i - v_j)] +
// 7/2 m_j A_j / r (without G), with aux[j] = (A_j, Phi_j) published by pass
// 1 (G included) and ai = the target's own. Zero separations contribute 0.
template <class T, class T4, int UNROLL, class Pos>
__device__ __forceinline__ void eih_terms(const Pos& sep, const T4* __restrict__ vs, const T4* __restrict__ aux,
                                          int n, int j0, int js, T4 vi, T4 ai, T3<T>& S) {
    T sx = T(0), sy = T(0), sz = T(0);
#pragma unroll UNROLL
    for (int j = j0; j < n; j += js) {
        T dx, dy, dz, mj, inv;
        sep(j, dx, dy, dz, mj, inv);
        const T4 vj = vs[j], aj = aux[j];
        const T inv2 = inv * inv;
        const T vij = vi.x * vj.x + vi.y * vj.y + vi.z * vj.z;
        const T dvi = dx * vi.x + dy * vi.y + dz * vi.z;   // d.v_i = -r n.v_i
        const T dvj = dx * vj.x + dy * vj.y + dz * vj.z;
        const T dA = dx * aj.x + dy * aj.y + dz * aj.z;
        const T nvj = dvj * inv;
        const T B = T(-4) * ai.w - aj.w + vi.w + T(2) * vj.w - T(4) * vij - T(1.5) * nvj * nvj + T(0.5) * dA;
        const T W = (T(3) * dvj - T(4) * dvi) * inv;
        const T f = mj * inv2, fb = f * inv * B, g7 = T(3.5) * mj * inv;
        sx += fb * dx + f * W * (vi.x - vj.x) + g7 * aj.x;
        sy += fb * dy + f * W * (vi.y - vj.y) + g7 * aj.y;
        sz += fb * dz + f * W * (vi.z - vj.z) + g7 * aj.z;
    }
    S.x = sx; S.y = sy; S.z = sz;
}

// Separation, mass and inverse distance of source j from the target, FP32
// from the double-single slab (mixed) or FP64.
struct SepF32 {
    const EnsSlab<true>& s;
    float4 hi, lo;
    float eps2;
    __device__ __forceinline__ void operator()(int j, float& dx, float& dy, float& dz, float& mj, float& inv) const {
        const float4 h = s.hi[j], l = s.lo[j];
        dx = (h.x - hi.x) + (l.x - lo.x);
        dy = (h.y - hi.y) + (l.y - lo.y);
        dz = (h.z - hi.z) + (l.z - lo.z);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
        const float iv = rsqrt_approx(r2);
        inv = r2 > 0.f ? iv : 0.f;
        mj = h.w;
    }
};
struct SepF64 {
    const EnsSlab<false>& s;
    double4 xi;
    double eps2;
    __device__ __forceinline__ void operator()(int j, double& dx, double& dy, double& dz, double& mj,
                                               double& inv) const {
        const double4 xj = s.x[j];
        dx = xj.x - xi.x; dy = xj.y - xi.y; dz = xj.z - xi.z;
        const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
        inv = r2 > 0.0 ? rsqrt(r2) : 0.0;
        mj = xj.w;
    }
};

// Sum of the lps partial sums of the aligned lane groups (the sources of a
// body beyond the first 32 are split among lps lanes); afterwards lane s holds
// the total of group s (the owner of body 32 + s) when `own`.
__device__ __forceinline__ double group_total(double v, int lps, int lane, bool own) {
    for (int o = lps >> 1; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, own ? lane * lps : 0);
}

// Level-3 (EIH) accelerations of the warp's bodies lane and 32 + lane:
// pass 1 sums A and Phi of every body and publishes them to aux, pass 2 the
// EIH terms. a[q] = A + c^-2 G S (FP64 results; FP32 pair arithmetic when
// MIXED).
template <bool MIXED, int UNROLL>
__device__ __forceinline__ void eih_accel(const EnsSlab<MIXED>& slab, typename EnsAux<MIXED>::T4* aux, int n,
                                          int lane, bool two, bool v0, bool v1, bool sec, int sb, int sub, int lps,
                                          double eps2, double G, double c2, double a[2][3]) {
    using T = typename EnsAux<MIXED>::T;
    using T4 = typename EnsAux<MIXED>::T4;
    double A[2][4];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (q == 1 && !two) { A[1][0] = A[1][1] = A[1][2] = A[1][3] = 0.0; continue; }
        const int idx = q ? (sec ? 32 + sb : 0) : (v0 ? lane : 0);
        const int j0 = q ? sub : 0, js = q ? lps : 1;
        double sx, sy, sz, sp;
        if constexpr (MIXED) {
            float3 aN;
            float ph;
            newton_phi_f32<UNROLL>(slab, n, j0, js, slab.hi[idx], slab.lo[idx], (float)eps2, aN, ph);
            sx = aN.x; sy = aN.y; sz = aN.z; sp = ph;
        } else {
            double3 aN;
            newton_phi_f64<UNROLL>(slab, n, j0, js, slab.x[idx], eps2, aN, sp);
            sx = aN.x; sy = aN.y; sz = aN.z;
        }
        if (q == 1) {
            sx = group_total(sx, lps, lane, v1); sy = group_total(sy, lps, lane, v1);
            sz = group_total(sz, lps, lane, v1); sp = group_total(sp, lps, lane, v1);
        }
        A[q][0] = G * sx; A[q][1] = G * sy; A[q][2] = G * sz; A[q][3] = G * sp;
    }
    if (v0) aux[lane] = T4{(T)A[0][0], (T)A[0][1], (T)A[0][2], (T)A[0][3]};
    if (v1) aux[32 + lane] = T4{(T)A[1][0], (T)A[1][1], (T)A[1][2], (T)A[1][3]};
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (q == 1 && !two) { a[1][0] = a[1][1] = a[1][2] = 0.0; continue; }
        const int idx = q ? (sec ? 32 + sb : 0) : (v0 ? lane : 0);
        const int j0 = q ? sub : 0, js = q ? lps : 1;
        T3<T> S;
        if constexpr (MIXED)
            eih_terms<float, float4, UNROLL>(SepF32{slab, slab.hi[idx], slab.lo[idx], (float)eps2}, slab.v, aux, n,
                                             j0, js, slab.v[idx], aux[idx], S);
        else
            eih_terms<double, double4, UNROLL>(SepF64{slab, slab.x[idx], eps2}, slab.v, aux, n, j0, js,
                                               slab.v[idx], aux[idx], S);
        double sx = S.x, sy = S.y, sz = S.z;
        if (q == 1) {
            sx = group_total(sx, lps, lane, v1); sy = group_total(sy, lps, lane, v1);
            sz = group_total(sz, lps, lane, v1);
        }
        const double k = G * c2;
        a[q][0] = A[q][0] + k * sx; a[q][1] = A[q][1] + k * sy; a[q][2] = A[q][2] + k * sz;
    }
}

template <bool MIXED, int PNL, int UNROLL, int NST>
__global__ void k_ensemble(int32_t nsys, const int32_t* __restrict__ order, const int32_t* __restrict__ off,
                           double4* __restrict__ pm, double4* __restrict__ vel, double G, double eps2, PnK<double> pk,
                           Coeffs k, int64_t nsteps, int check_every, unsigned int* __restrict__ work,
                           const volatile int* __restrict__ cancel, int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char ens_smem[];
    EnsSlab<MIXED>& slab = reinterpret_cast<EnsSlab<MIXED>*>(ens_smem)[threadIdx.x >> 5];
    // level 3 only: 64 (A, Phi) records per warp after all the block's slabs
    using Aux4 = typename EnsAux<MIXED>::T4;
    Aux4* aux = reinterpret_cast<Aux4*>(ens_smem + (blockDim.x >> 5) * sizeof(EnsSlab<MIXED>)) +
                (threadIdx.x >> 5) * 64;
    const int lane = threadIdx.x & 31;
    const float Gf = (float)G, epsf = (float)eps2;
    const PnK<float> pkf = pn_float(pk);
    for (;;) {
        unsigned int w = 0;
        if (lane == 0) w = atomicAdd(work, 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= (unsigned)nsys) break;
        const int sys = order[w];
        const int b0 = off[sys], n = off[sys + 1] - b0;
        const bool two = n > 32;
        const bool v0 = lane < n, v1 = lane + 32 < n;
        // the r = n - 32 bodies beyond the first 32 get lps lanes each (the
        // largest power of two with lps * r <= 32), which split its sources
        const int r = two ? n - 32 : 0;
        int lps = 32;
        while (lps > 1 && lps * r > 32) lps >>= 1;
        const int sb = lane / lps, sub = lane & (lps - 1);
        const bool sec = two && sb < r;
        double4 x[2], v[2];
        x[0] = v0 ? pm[b0 + lane] : make_double4(0, 0, 0, 0);
        v[0] = v0 ? vel[b0 + lane] : make_double4(0, 0, 0, 0);
        x[1] = v1 ? pm[b0 + lane + 32] : make_double4(0, 0, 0, 0);
        v[1] = v1 ? vel[b0 + lane + 32] : make_double4(0, 0, 0, 0);
        bool stop = false;
        for (int64_t step = 0; step < nsteps; ++step) {
            if (step % check_every == 0) {
                int cflag = 0;
                if (lane == 0) cflag = *cancel;
                cflag = __shfl_sync(0xffffffffu, cflag, 0);
                if (cflag) {
                    if (lane == 0) atomicOr(err, ASTER_DEVERR_CANCEL);
                    stop = true;
                    break;
                }
            }
#pragma unroll
            for (int st = 0; st < NST; ++st) {  // unrolled: coefficients stay in registers
                const double c = k.cdt[st], d = k.ddt[st];
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    x[q].x += c * v[q].x; x[q].y += c * v[q].y; x[q].z += c * v[q].z;
                    const bool vq = q ? v1 : v0;
                    if (!vq) continue;
                    const int idx = lane + 32 * q;
                    const double vsq = v[q].x * v[q].x + v[q].y * v[q].y + v[q].z * v[q].z;
                    if (MIXED) {
                        EnsSlab<true>& sl = reinterpret_cast<EnsSlab<true>&>(slab);
                        float4 h, l;
                        ds_split(x[q].x, h.x, l.x);
                        ds_split(x[q].y, h.y, l.y);
                        ds_split(x[q].z, h.z, l.z);
                        h.w = (float)x[q].w;
                        l.w = 0.f;
                        sl.hi[idx] = h;
                        sl.lo[idx] = l;
                        sl.v[idx] = make_float4((float)v[q].x, (float)v[q].y, (float)v[q].z, (float)vsq);
                    } else {
                        EnsSlab<false>& sl = reinterpret_cast<EnsSlab<false>&>(slab);
                        sl.x[idx] = x[q];
                        sl.v[idx] = make_double4(v[q].x, v[q].y, v[q].z, vsq);
                    }
                }
                __syncwarp();
                double a[2][3];
                if constexpr (PNL == 3) {
                    eih_accel<MIXED, UNROLL>(slab, aux, n, lane, two, v0, v1, sec, sb, sub, lps, eps2, G, pk.c2, a);
                } else {
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    if (q == 1 && !two) { a[1][0] = a[1][1] = a[1][2] = 0.0; continue; }
                    // body `lane` (q = 0, all sources); for q = 1 body 32 + sb, its
                    // sources split among the lps lanes of group sb
                    const int idx = q ? (sec ? 32 + sb : 0) : (v0 ? lane : 0);  // idle slots read body 0
                    const int j0 = q ? sub : 0, js = q ? lps : 1;
                    double sx, sy, sz;
                    if (MIXED) {
                        const EnsSlab<true>& sl = reinterpret_cast<const EnsSlab<true>&>(slab);
                        float3 aN, a1, a2;
                        accel_f32<PNL, UNROLL>(sl, n, j0, js, sl.hi[idx], sl.lo[idx], sl.v[idx], epsf, Gf, pkf, aN,
                                               a1, a2);
                        sx = ((double)aN.x + (double)a1.x) + (double)a2.x;
                        sy = ((double)aN.y + (double)a1.y) + (double)a2.y;
                        sz = ((double)aN.z + (double)a1.z) + (double)a2.z;
                    } else {
                        const EnsSlab<false>& sl = reinterpret_cast<const EnsSlab<false>&>(slab);
                        accel_f64<PNL, UNROLL>(sl, n, j0, js, sl.x[idx], sl.v[idx], eps2, G, pk, sx, sy, sz);
                    }
                    if (q == 1) {
                        // add the lps partial sums (aligned lane groups), then lane s
                        // (owner of body 32 + s) takes its group's total
                        for (int o = lps >> 1; o >= 1; o >>= 1) {
                            sx += __shfl_xor_sync(0xffffffffu, sx, o);
                            sy += __shfl_xor_sync(0xffffffffu, sy, o);
                            sz += __shfl_xor_sync(0xffffffffu, sz, o);
                        }
                        const int src = v1 ? lane * lps : 0;
                        sx = __shfl_sync(0xffffffffu, sx, src);
                        sy = __shfl_sync(0xffffffffu, sy, src);
                        sz = __shfl_sync(0xffffffffu, sz, src);
                    }
                    a[q][0] = G * sx; a[q][1] = G * sy; a[q][2] = G * sz;
                }
                }
                __syncwarp();
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    v[q].x += d * a[q][0]; v[q].y += d * a[q][1]; v[q].z += d * a[q][2];
                }
            }
            const double c = k.cdt[NST];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                x[q].x += c * v[q].x; x[q].y += c * v[q].y; x[q].z += c * v[q].z;
            }
        }
        if (v0) { pm[b0 + lane] = x[0]; vel[b0 + lane] = v[0]; }
        if (v1) { pm[b0 + lane + 32] = x[1]; vel[b0 + lane + 32] = v[1]; }
        if (stop) break;
    }
}

// FP64 energy of one system per warp: Newtonian, plus (pn) the 1PN energy of
// the EIH Lagrangian. Its G^2 term is (1/2) sum_a m_a Phi_a^2; for the
// pairwise law (eih = 0) only its two-body part, sum over pairs of
// G^2 m_i m_j (m_i + m_j) / (2 r^2), is kept.
__global__ void k_ensemble_energy(int32_t nsys, const int32_t* __restrict__ off, const double4* __restrict__ pm,
                                  const double4* __restrict__ vel, double G, double eps2, double inv_c2, int pn,
                                  int eih, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t sys = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (sys >= nsys) return;
    const int b0 = off[sys], n = off[sys + 1] - b0;
    double e = 0.0, e1 = 0.0;
    for (int i = lane; i < n; i += 32) {
        const double4 xi = pm[b0 + i], vi = vel[b0 + i];
        const double v2 = vi.x * vi.x + vi.y * vi.y + vi.z * vi.z;
        e += 0.5 * xi.w * v2;
        e1 += 0.375 * xi.w * v2 * v2;
        if (pn && eih) {
            double phi = 0.0;
            for (int j = 0; j < n; ++j) {
                if (j == i) continue;
                const double4 xj = pm[b0 + j];
                const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
                phi += G * xj.w / sqrt(dx * dx + dy * dy + dz * dz + eps2);
            }
            e1 += 0.5 * xi.w * phi * phi;
        }
        for (int j = i + 1; j < n; ++j) {
            const double4 xj = pm[b0 + j], vj = vel[b0 + j];
            const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            const double r = sqrt(dx * dx + dy * dy + dz * dz + eps2);
            e -= G * xi.w * xj.w / r;
            const double vj2 = vj.x * vj.x + vj.y * vj.y + vj.z * vj.z;
            const double vij = vi.x * vj.x + vi.y * vj.y + vi.z * vj.z;
            const double nvi = (dx * vi.x + dy * vi.y + dz * vi.z) / r;
            const double nvj = (dx * vj.x + dy * vj.y + dz * vj.z) / r;
            e1 += G * xi.w * xj.w / (2.0 * r) * (3.0 * (v2 + vj2) - 7.0 * vij - nvi * nvj);
            if (!eih) e1 += G * G * xi.w * xj.w * (xi.w + xj.w) / (2.0 * r * r);
        }
    }
    double t = e + (pn ? inv_c2 * e1 : 0.0);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) out[sys] = t;
}

__global__ void k_pack_ens(int64_t n, const double* __restrict__ pos, const double* __restrict__ vel,
                           const double* __restrict__ m, double4* __restrict__ pm, double4* __restrict__ v4,
                           int* __restrict__ err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2], mm = m[i];
        const double vx = vel ? vel[3 * i] : 0.0, vy = vel ? vel[3 * i + 1] : 0.0, vz = vel ? vel[3 * i + 2] : 0.0;
        if (!(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(mm) && isfinite(vx) && isfinite(vy) &&
              isfinite(vz)))
            atomicOr(err, ASTER_DEVERR_NONFINITE);
        pm[i] = make_double4(x, y, z, mm);
        v4[i] = make_double4(vx, vy, vz, 0.0);
    }
}

__global__ void k_unpack_ens(int64_t n, const double4* __restrict__ src, double* __restrict__ dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 v = src[i];
        dst[3 * i] = v.x; dst[3 * i + 1] = v.y; dst[3 * i + 2] = v.z;
    }
}

template <bool MIXED, int PNL, int UNROLL>
int launch_ensemble(aster_ctx* c, const aster_params* p, const Coeffs& k, int64_t nsteps, int wpb, int check_every,
                    bool use_graph) {
    EnsBufs& e = c->ens;
    auto kern = k.nst == 3 ? k_ensemble<MIXED, PNL, UNROLL, 3> : k_ensemble<MIXED, PNL, UNROLL, 1>;
    const size_t smem = (size_t)wpb * (sizeof(EnsSlab<MIXED>) +
                                       (PNL == 3 ? 64 * sizeof(typename EnsAux<MIXED>::T4) : 0));
    if (smem > 48 * 1024) ASTER_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    ASTER_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpb * 32, smem));
    if (per_sm < 1) return ASTER_ERR_UNSUPPORTED;
    int64_t blocks = (int64_t)c->sm_count * per_sm;
    const int64_t need = (e.nsys + wpb - 1) / wpb;
    if (blocks > need) blocks = need;
    const PnK<double> pk = make_pn(p);
    unsigned int* work = e.counter.as<unsigned int>();
    auto enqueue = [&](cudaStream_t s) -> int {
        ASTER_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned int), s));
        kern<<<(unsigned)blocks, wpb * 32, smem, s>>>(e.nsys, e.order.as<int32_t>(), e.off.as<int32_t>(),
                                                     e.pm.as<double4>(), e.vel.as<double4>(), p->G, p->eps2, pk, k,
                                                     nsteps, check_every, work, e.cancel_dev, c->err_dev);
        ASTER_CUDA(cudaGetLastError());
        return ASTER_OK;
    };
    if (!use_graph) return enqueue(c->stream);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ASTER_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int st = enqueue(c->stream);
    cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (st != ASTER_OK) { if (graph) cudaGraphDestroy(graph); return st; }
    if (ce != cudaSuccess) return aster_cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return aster_cuda_fail(ce, "cudaGraphInstantiate", __FILE__, __LINE__);
    ce = cudaGraphLaunch(exec, c->stream);
    // the executable graph may be destroyed once its launch is enqueued
    cudaGraphExecDestroy(exec);
    if (ce != cudaSuccess) return aster_cuda_fail(ce, "cudaGraphLaunch", __FILE__, __LINE__);
    return ASTER_OK;
}

template <bool MIXED, int PNL>
int dispatch_unroll(aster_ctx* c, const aster_params* p, const Coeffs& k, int64_t nsteps, int wpb, int unroll,
                    int check_every, bool g) {
    switch (unroll) {
        case 1: return launch_ensemble<MIXED, PNL, 1>(c, p, k, nsteps, wpb, check_every, g);
        case 4: return launch_ensemble<MIXED, PNL, 4>(c, p, k, nsteps, wpb, check_every, g);
        default: return launch_ensemble<MIXED, PNL, 2>(c, p, k, nsteps, wpb, check_every, g);
    }
}

// The ensemble's force law: ASTER_EIH (with ASTER_PN1, and neither 2PN nor
// 2.5PN) selects level 3; the other bits are checked as everywhere else.
int ens_check_params(const aster_params* p, int* level) {
    if (!p) return ASTER_ERR_INVALID_ARG;
    aster_params q = *p;
    const bool eih = (q.force_law & ASTER_EIH) != 0;
    q.force_law &= ~ASTER_EIH;
    ASTER_TRY(aster_check_params(&q));
    if (eih && (!(q.force_law & ASTER_PN1) || (q.force_law & (ASTER_PN2 | ASTER_PN25)))) return ASTER_ERR_UNSUPPORTED;
    *level = eih ? 3 : pn_level(&q);
    return ASTER_OK;
}

}  // namespace

extern "C" int aster_ensemble_upload(aster_ctx* c, int32_t nsys, const int64_t* offsets, const double* pos,
                                     const double* vel, const double* mass) {
    if (!c || nsys <= 0 || !offsets || !pos || !mass) return ASTER_ERR_INVALID_ARG;
    if (offsets[0] != 0) return ASTER_ERR_INVALID_ARG;
    std::vector<int32_t> off32(nsys + 1);
    for (int32_t s = 0; s < nsys; ++s) {
        const int64_t sz = offsets[s + 1] - offsets[s];
        if (sz < 1) return ASTER_ERR_INVALID_ARG;
        if (sz > ASTER_ENSEMBLE_MAX_BODIES) return ASTER_ERR_TOO_LARGE;
    }
    const int64_t nb = offsets[nsys];
    if (nb > (int64_t)INT32_MAX) return ASTER_ERR_TOO_LARGE;
    double pairs = 0.0;
    for (int32_t s = 0; s <= nsys; ++s) off32[s] = (int32_t)offsets[s];
    std::vector<int32_t> order(nsys);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return off32[a + 1] - off32[a] > off32[b + 1] - off32[b];
    });
    for (int32_t s = 0; s < nsys; ++s) {
        const double sz = (double)(off32[s + 1] - off32[s]);
        pairs += sz * (sz - 1.0);
    }
    ASTER_TRY(aster_begin(c));
    EnsBufs& e = c->ens;
    ASTER_TRY(e.pm.ensure((size_t)nb * sizeof(double4)));
    ASTER_TRY(e.vel.ensure((size_t)nb * sizeof(double4)));
    ASTER_TRY(e.off.ensure((size_t)(nsys + 1) * 4));
    ASTER_TRY(e.order.ensure((size_t)nsys * 4));
    ASTER_TRY(e.counter.ensure(256));
    if (!e.cancel_host) {
        void* h = nullptr;
        ASTER_CUDA(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped));
        e.cancel_host = static_cast<volatile int*>(h);
        *e.cancel_host = 0;
        void* d = nullptr;
        ASTER_CUDA(cudaHostGetDevicePointer(&d, h, 0));
        e.cancel_dev = static_cast<int*>(d);
    }
    const size_t v3 = (size_t)nb * 3 * sizeof(double);
    ASTER_TRY(c->stage.ensure(2 * v3 + (size_t)nb * sizeof(double)));
    double* sp = c->stage.as<double>();
    double* sv = sp + 3 * nb;
    double* sm = sv + 3 * nb;
    ASTER_CUDA(cudaMemcpyAsync(sp, pos, v3, cudaMemcpyHostToDevice, c->stream));
    if (vel) ASTER_CUDA(cudaMemcpyAsync(sv, vel, v3, cudaMemcpyHostToDevice, c->stream));
    ASTER_CUDA(cudaMemcpyAsync(sm, mass, (size_t)nb * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    ASTER_CUDA(cudaMemcpyAsync(e.off.ptr, off32.data(), (size_t)(nsys + 1) * 4, cudaMemcpyHostToDevice, c->stream));
    ASTER_CUDA(cudaMemcpyAsync(e.order.ptr, order.data(), (size_t)nsys * 4, cudaMemcpyHostToDevice, c->stream));
    const int grid = (int)std::min<int64_t>((nb + 255) / 256, (int64_t)c->sm_count * 16);
    k_pack_ens<<<grid, 256, 0, c->stream>>>(nb, sp, vel ? sv : nullptr, sm, e.pm.as<double4>(), e.vel.as<double4>(),
                                            c->err_dev);
    ASTER_CUDA(cudaGetLastError());
    int st = aster_finish(c);  // host vectors must outlive the copies: synchronised here
    if (st != ASTER_OK) return st;
    e.nsys = nsys;
    e.nbodies = nb;
    e.pair_evals_per_stage = pairs;
    return ASTER_OK;
}

extern "C" int aster_ensemble_download(aster_ctx* c, double* pos, double* vel) {
    if (!c) return ASTER_ERR_INVALID_ARG;
    EnsBufs& e = c->ens;
    if (e.nsys <= 0) return ASTER_ERR_NO_STATE;
    ASTER_CUDA(cudaSetDevice(c->device));
    const int64_t nb = e.nbodies;
    const size_t v3 = (size_t)nb * 3 * sizeof(double);
    ASTER_TRY(c->stage.ensure(2 * v3));
    double* st = c->stage.as<double>();
    const int grid = (int)std::min<int64_t>((nb + 255) / 256, (int64_t)c->sm_count * 16);
    if (pos) {
        k_unpack_ens<<<grid, 256, 0, c->stream>>>(nb, e.pm.as<double4>(), st);
        ASTER_CUDA(cudaGetLastError());
        ASTER_CUDA(cudaMemcpyAsync(pos, st, v3, cudaMemcpyDeviceToHost, c->stream));
    }
    if (vel) {
        k_unpack_ens<<<grid, 256, 0, c->stream>>>(nb, e.vel.as<double4>(), st + 3 * nb);
        ASTER_CUDA(cudaGetLastError());
        ASTER_CUDA(cudaMemcpyAsync(vel, st + 3 * nb, v3, cudaMemcpyDeviceToHost, c->stream));
    }
    ASTER_CUDA(cudaStreamSynchronize(c->stream));
    return ASTER_OK;
}

extern "C" int aster_ensemble_run(aster_ctx* c, const aster_params* p, int integrator, int precision, int64_t nsteps,
                                  const aster_ensemble_config* cfg) {
    if (!c || nsteps < 0) return ASTER_ERR_INVALID_ARG;
    int pnl = 0;
    ASTER_TRY(ens_check_params(p, &pnl));
    if (c->ens.nsys <= 0) return ASTER_ERR_NO_STATE;
    if (integrator != ASTER_INTEGRATOR_LEAPFROG && integrator != ASTER_INTEGRATOR_YOSHIDA4) return ASTER_ERR_INVALID_ARG;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    int wpb = cfg && cfg->warps_per_block ? cfg->warps_per_block : 4;
    int unroll = cfg && cfg->unroll ? cfg->unroll : 2;
    int check = cfg && cfg->check_every ? cfg->check_every : 256;
    // stream capture is not possible on the legacy default stream
    bool graph = (cfg ? cfg->use_graph != 0 : true) && c->stream != nullptr;
    if (wpb < 1 || wpb > 16 || (unroll != 1 && unroll != 2 && unroll != 4) || check < 1) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    *c->ens.cancel_host = 0;
    const Coeffs k = make_coeffs(integrator, p->dt);
    // PN level: 3 EIH; 2 when a 2PN or 2.5PN term is requested, else 1 for 1PN alone
    cudaEventRecord(c->ev[0], c->stream);
    int st;
    if (precision == ASTER_MIXED)
        st = pnl == 3 ? dispatch_unroll<true, 3>(c, p, k, nsteps, wpb, unroll, check, graph)
           : pnl == 2 ? dispatch_unroll<true, 2>(c, p, k, nsteps, wpb, unroll, check, graph)
           : pnl == 1 ? dispatch_unroll<true, 1>(c, p, k, nsteps, wpb, unroll, check, graph)
                      : dispatch_unroll<true, 0>(c, p, k, nsteps, wpb, unroll, check, graph);
    else
        st = pnl == 3 ? dispatch_unroll<false, 3>(c, p, k, nsteps, wpb, unroll, check, graph)
           : pnl == 2 ? dispatch_unroll<false, 2>(c, p, k, nsteps, wpb, unroll, check, graph)
           : pnl == 1 ? dispatch_unroll<false, 1>(c, p, k, nsteps, wpb, unroll, check, graph)
                      : dispatch_unroll<false, 0>(c, p, k, nsteps, wpb, unroll, check, graph);
    if (st != ASTER_OK) return st;
    cudaEventRecord(c->ev[1], c->stream);
    st = aster_finish(c);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = c->stats.ms_force = ms;
    c->stats.kernels = 1;
    c->stats.interactions = c->ens.pair_evals_per_stage * k.nst * (double)nsteps;
    return st;
}

extern "C" int aster_ensemble_energy(aster_ctx* c, const aster_params* p, double* energy) {
    if (!c || !energy) return ASTER_ERR_INVALID_ARG;
    int pnl = 0;
    ASTER_TRY(ens_check_params(p, &pnl));
    EnsBufs& e = c->ens;
    if (e.nsys <= 0) return ASTER_ERR_NO_STATE;
    ASTER_TRY(aster_begin(c));
    ASTER_TRY(c->scratch.ensure((size_t)e.nsys * sizeof(double)));
    const int wpb = 4;
    const int blocks = (e.nsys + wpb - 1) / wpb;
    const bool pn = (p->force_law & ASTER_PN1) != 0;
    k_ensemble_energy<<<blocks, wpb * 32, 0, c->stream>>>(e.nsys, e.off.as<int32_t>(), e.pm.as<double4>(),
                                                           e.vel.as<double4>(), p->G, p->eps2,
                                                           pn ? 1.0 / (p->c * p->c) : 0.0, pn ? 1 : 0,
                                                           pnl == 3 ? 1 : 0, c->scratch.as<double>());
    ASTER_CUDA(cudaGetLastError());
    ASTER_CUDA(cudaMemcpyAsync(energy, c->scratch.ptr, (size_t)e.nsys * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream));
    return aster_finish(c);
}

extern "C" int aster_ensemble_cancel(aster_ctx* c) {
    if (!c || !c->ens.cancel_host) return ASTER_ERR_INVALID_ARG;
    *c->ens.cancel_host = 1;
    return ASTER_OK;
}
