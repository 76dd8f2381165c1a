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
// sums the bracketed terms. Sources at zero separation (the target itself,
// or a body at exactly its position) are left out of both sums, softened or
// not. For two unsoftened bodies it equals get_pn1.
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
// Mixed slab, pair-interleaved: element k of each array holds bodies 2k and
// 2k + 1, so that every paired FP32 operand is one aligned register pair
// (positions double-single, hi + lo). Bodies past the system's size hold
// zeros (zero mass), so a half-used last pair contributes nothing.
template <>
struct EnsSlab<true> {
    float4 A[32];  // (x_hi, x_hi', y_hi, y_hi')   ' = the odd body of the pair
    float4 B[32];  // (z_hi, z_hi', m, m')
    float4 C[32];  // (x_lo, x_lo', y_lo, y_lo')
    float4 D[32];  // (z_lo, z_lo', vz, vz')
    float4 E[32];  // (vx, vx', vy, vy')
    float2 F[32];  // (|v|^2, |v'|^2)
};
template <>
struct EnsSlab<false> {
    double4 x[64];  // (x, y, z, m)
    double4 v[64];  // (vx, vy, vz, |v|^2)
};

// Float index of body b's half in a pair-interleaved float4 array (its x
// half; the y half is 2 further on).
__device__ __forceinline__ int pslot(int b) { return ((b >> 1) << 2) | (b & 1); }

// One body of the mixed slab as scalars.
struct BodyF32 {
    float hx, hy, hz, m, lx, ly, lz, vx, vy, vz, w;
};
__device__ __forceinline__ BodyF32 slab_body(const EnsSlab<true>& s, int b) {
    const float* A = reinterpret_cast<const float*>(s.A);
    const float* B = reinterpret_cast<const float*>(s.B);
    const float* C = reinterpret_cast<const float*>(s.C);
    const float* D = reinterpret_cast<const float*>(s.D);
    const float* E = reinterpret_cast<const float*>(s.E);
    const float* F = reinterpret_cast<const float*>(s.F);
    const int o = pslot(b);
    return BodyF32{A[o], A[o + 2], B[o], B[o + 2], C[o], C[o + 2], D[o], E[o], E[o + 2], D[o + 2], F[b]};
}
__device__ __forceinline__ void slab_put(EnsSlab<true>& s, int b, const double4& x, const double4& v) {
    float* A = reinterpret_cast<float*>(s.A);
    float* B = reinterpret_cast<float*>(s.B);
    float* C = reinterpret_cast<float*>(s.C);
    float* D = reinterpret_cast<float*>(s.D);
    float* E = reinterpret_cast<float*>(s.E);
    float* F = reinterpret_cast<float*>(s.F);
    const int o = pslot(b);
    float h, l;
    ds_split(x.x, h, l); A[o] = h; C[o] = l;
    ds_split(x.y, h, l); A[o + 2] = h; C[o + 2] = l;
    ds_split(x.z, h, l); B[o] = h; D[o] = l;
    B[o + 2] = (float)x.w;
    D[o + 2] = (float)v.z;
    E[o] = (float)v.x;
    E[o + 2] = (float)v.y;
    F[b] = (float)(v.x * v.x + v.y * v.y + v.z * v.z);
}

// Per target: minus its double-single position, broadcast to both halves.
struct TargetX2 {
    float2 nhx, nhy, nhz, nlx, nly, nlz;
    __device__ __forceinline__ explicit TargetX2(const BodyF32& t)
        : nhx(make_float2(-t.hx, -t.hx)), nhy(make_float2(-t.hy, -t.hy)), nhz(make_float2(-t.hz, -t.hz)),
          nlx(make_float2(-t.lx, -t.lx)), nly(make_float2(-t.ly, -t.ly)), nlz(make_float2(-t.lz, -t.lz)) {}
    // d = x_j - x_i for the pair in slot q: (h_j - h_i) + (l_j - l_i)
    __device__ __forceinline__ void sep(const EnsSlab<true>& s, int q, float2& dx, float2& dy, float2& dz) const {
        const float4 a = s.A[q], b = s.B[q], c = s.C[q], d = s.D[q];
        dx = __fadd2_rn(__fadd2_rn(make_float2(a.x, a.y), nhx), __fadd2_rn(make_float2(c.x, c.y), nlx));
        dy = __fadd2_rn(__fadd2_rn(make_float2(a.z, a.w), nhy), __fadd2_rn(make_float2(c.z, c.w), nly));
        dz = __fadd2_rn(__fadd2_rn(make_float2(b.x, b.y), nhz), __fadd2_rn(make_float2(d.x, d.y), nlz));
    }
};

// r^-1 of both halves; a zero r^2 (the target itself, unsoftened) gives 0.
__device__ __forceinline__ float2 inv_r_x2(const float2 dx, const float2 dy, const float2 dz, const float2 eps2) {
    float2 r2 = __ffma2_rn(dz, dz, eps2);
    r2 = __ffma2_rn(dy, dy, r2);
    r2 = __ffma2_rn(dx, dx, r2);
    float2 inv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    inv.x = r2.x > 0.f ? inv.x : 0.f;
    inv.y = r2.y > 0.f ? inv.y : 0.f;
    return inv;
}

// EIH form: r^-1 with r^2 = |d|^2 + eps2, 0 where d itself is zero. With
// softening the target's own slot has r^2 = eps2 > 0; its potential m / r and
// 7/2 m A / r terms must not count, so the guard is on |d|^2.
__device__ __forceinline__ float2 inv_r_x2_nz(const float2 dx, const float2 dy, const float2 dz, const float2 eps2) {
    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    const float2 r2 = __fadd2_rn(d2, eps2);
    float2 inv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    inv.x = d2.x > 0.f ? inv.x : 0.f;
    inv.y = d2.y > 0.f ? inv.y : 0.f;
    return inv;
}

// Mixed accelerations of target t (without G): sums over the source pairs
// q = q0, q0 + qs, ... < np (qs > 1: the lanes that share a target split its
// sources). Two sources per paired FP32 instruction at every level: Newton,
// Newton + 1PN (newton_pn1_x2) and level 2, any of 1PN/2PN/2.5PN by flags
// (newton_pn_all_x2). The Newtonian, 1PN and 2PN + 2.5PN sums are kept apart.
template <int PNL, int UNROLL>
__device__ __forceinline__ void accel_f32(const EnsSlab<true>& s, int np, int q0, int qs, const BodyF32& t,
                                          float eps2, float G, const PnK<float>& k, float3& aN, float3& a1,
                                          float3& a2) {
    const TargetX2 tx(t);
    const float2 e2 = make_float2(eps2, eps2);
    float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax, px = ax, py = ax, pz = ax;
    float qx = 0.f, qy = 0.f, qz = 0.f;
    if constexpr (PNL == 0) {
#pragma unroll UNROLL
        for (int q = q0; q < np; q += qs) {
            float2 dx, dy, dz;
            tx.sep(s, q, dx, dy, dz);
            const float4 b = s.B[q];
            const float2 inv = inv_r_x2(dx, dy, dz, e2);
            const float2 sN = __fmul2_rn(__fmul2_rn(make_float2(b.z, b.w), inv), __fmul2_rn(inv, inv));
            ax = __ffma2_rn(dx, sN, ax);
            ay = __ffma2_rn(dy, sN, ay);
            az = __ffma2_rn(dz, sN, az);
        }
    } else if constexpr (PNL == 1) {
        const float2 vix = make_float2(t.vx, t.vx), viy = make_float2(t.vy, t.vy), viz = make_float2(t.vz, t.vz);
        const float2 vi4x = make_float2(4.f * t.vx, 4.f * t.vx), vi4y = make_float2(4.f * t.vy, 4.f * t.vy),
                     vi4z = make_float2(4.f * t.vz, 4.f * t.vz);
        const float2 nvi2 = make_float2(-t.w, -t.w), mi5G = make_float2(5.f * G * t.m, 5.f * G * t.m);
        const float2 G4 = make_float2(4.f * G, 4.f * G);
#pragma unroll UNROLL
        for (int q = q0; q < np; q += qs) {
            float2 dx, dy, dz;
            tx.sep(s, q, dx, dy, dz);
            const float4 b = s.B[q], d = s.D[q], e = s.E[q];
            newton_pn1_x2<true>(dx, dy, dz, make_float2(b.z, b.w), make_float2(e.x, e.y), make_float2(e.z, e.w),
                                make_float2(d.z, d.w), s.F[q], vix, viy, viz, vi4x, vi4y, vi4z, nvi2, mi5G, e2, G4,
                                ax, ay, az, px, py, pz);
        }
        const float mc2 = -k.c2;  // the 1PN term is -c^-2 times newton_pn1_x2's sum
        px = __fmul2_rn(px, make_float2(mc2, mc2));
        py = __fmul2_rn(py, make_float2(mc2, mc2));
        pz = __fmul2_rn(pz, make_float2(mc2, mc2));
    } else {  // the flagged PN terms, two sources per paired instruction as well
        const float2 vix = make_float2(t.vx, t.vx), viy = make_float2(t.vy, t.vy), viz = make_float2(t.vz, t.vz);
        const float2 vi4x = make_float2(4.f * t.vx, 4.f * t.vx), vi4y = make_float2(4.f * t.vy, 4.f * t.vy),
                     vi4z = make_float2(4.f * t.vz, 4.f * t.vz);
        const float2 nvi2 = make_float2(-t.w, -t.w), vi2 = make_float2(t.w, t.w);
        const float2 mi5G = make_float2(5.f * G * t.m, 5.f * G * t.m), Gmi = make_float2(G * t.m, G * t.m);
        const float2 G4 = make_float2(4.f * G, 4.f * G), G2 = make_float2(G, G);
        const float2 nk = make_float2(-0.8f * k.ic, -0.8f * k.ic);
        float2 q2x = make_float2(0.f, 0.f), q2y = q2x, q2z = q2x;
#pragma unroll UNROLL
        for (int q = q0; q < np; q += qs) {
            float2 dx, dy, dz;
            tx.sep(s, q, dx, dy, dz);
            const float4 b = s.B[q], d = s.D[q], e = s.E[q];
            newton_pn_all_x2<true>(dx, dy, dz, make_float2(b.z, b.w), make_float2(e.x, e.y), make_float2(e.z, e.w),
                                   make_float2(d.z, d.w), s.F[q], vix, viy, viz, vi4x, vi4y, vi4z, nvi2, vi2, mi5G,
                                   Gmi, e2, G4, G2, nk, k.f, ax, ay, az, px, py, pz, q2x, q2y, q2z);
        }
        const float mc2 = -k.c2, mc4 = -k.c4;  // P and Q as newton_pn_all_x2 defines them
        px = __fmul2_rn(px, make_float2(mc2, mc2));
        py = __fmul2_rn(py, make_float2(mc2, mc2));
        pz = __fmul2_rn(pz, make_float2(mc2, mc2));
        qx = mc4 * (q2x.x + q2x.y);
        qy = mc4 * (q2y.x + q2y.y);
        qz = mc4 * (q2z.x + q2z.y);
    }
    aN = make_float3(ax.x + ax.y, ay.x + ay.y, az.x + az.y);
    a1 = make_float3(px.x + px.y, py.x + py.y, pz.x + pz.y);
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
// (both without G), mixed: source pairs q = q0, q0 + qs, ... < np.
template <int UNROLL>
__device__ __forceinline__ void newton_phi_f32(const EnsSlab<true>& s, int np, int q0, int qs, const BodyF32& t,
                                               float eps2, float3& aN, float& phi) {
    const TargetX2 tx(t);
    const float2 e2 = make_float2(eps2, eps2);
    float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax, ph = ax;
#pragma unroll UNROLL
    for (int q = q0; q < np; q += qs) {
        float2 dx, dy, dz;
        tx.sep(s, q, dx, dy, dz);
        const float4 b = s.B[q];
        const float2 inv = inv_r_x2_nz(dx, dy, dz, e2);
        const float2 mi = __fmul2_rn(make_float2(b.z, b.w), inv);
        const float2 sN = __fmul2_rn(mi, __fmul2_rn(inv, inv));
        ax = __ffma2_rn(dx, sN, ax);
        ay = __ffma2_rn(dy, sN, ay);
        az = __ffma2_rn(dz, sN, az);
        ph = __fadd2_rn(ph, mi);
    }
    aN = make_float3(ax.x + ax.y, ay.x + ay.y, az.x + az.y);
    phi = ph.x + ph.y;
}

template <int UNROLL>
__device__ __forceinline__ void newton_phi_f64(const EnsSlab<false>& s, int n, int j0, int js, double4 xi,
                                               double eps2, double3& aN, double& phi) {
    double ax = 0.0, ay = 0.0, az = 0.0, ph = 0.0;
#pragma unroll UNROLL
    for (int j = j0; j < n; j += js) {
        const double4 xj = s.x[j];
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double d2 = fma(dx, dx, fma(dy, dy, dz * dz));
        const double inv = d2 > 0.0 ? rsqrt(d2 + eps2) : 0.0;  // not the target itself
        const double mi = xj.w * inv;
        const double sN = mi * inv * inv;
        ax = fma(dx, sN, ax); ay = fma(dy, sN, ay); az = fma(dz, sN, az);
        ph += mi;
    }
    aN = make_double3(ax, ay, az);
    phi = ph;
}

// EIH pass 2 (level 3): sum over j of m_j / r^2 [d/r B + W (v_i - v_j)] +
// 7/2 m_j A_j / r (without G), with A_j and Phi_j (G included) from pass 1.
// Zero separations contribute 0. Mixed: source pairs q = q0, q0 + qs, ... < np
// of the pair-interleaved slab; pass 1 publishes A'_j = A_j / 2 and
// Q_j = 2 |v_j|^2 - Phi_j, aux = (A'_x, A'_x', A'_y, A'_y') in auxA and
// (A'_z, A'_z', Q, Q') in auxB; per target Ki = -4 Phi_i + |v_i|^2 =
// 4 Q_i - 7 |v_i|^2. With these B = Ki + Q_j - 4 v_i.v_j - 3/2 (d.v_j / r)^2
// + d.A'_j, and with k3 = m_j / r^3 the three terms are k3 B d,
// k3 (3 d.v_j - 4 d.v_i) (v_i - v_j) and 7 (m_j / r) A'_j.
template <int UNROLL>
__device__ __forceinline__ void eih_terms_f32(const EnsSlab<true>& s, const float4* __restrict__ auxA,
                                              const float4* __restrict__ auxB, int np, int q0, int qs,
                                              const BodyF32& t, float Q_i, float eps2, float3& S) {
    const TargetX2 tx(t);
    const float2 e2 = make_float2(eps2, eps2);
    const float2 vix = make_float2(t.vx, t.vx), viy = make_float2(t.vy, t.vy), viz = make_float2(t.vz, t.vz);
    const float2 n4x = make_float2(-4.f * t.vx, -4.f * t.vx), n4y = make_float2(-4.f * t.vy, -4.f * t.vy),
                 n4z = make_float2(-4.f * t.vz, -4.f * t.vz);  // -4 v_i
    const float ki = fmaf(4.f, Q_i, -7.f * t.w);
    const float2 Ki = make_float2(ki, ki);
    const float2 m1 = make_float2(-1.f, -1.f);
    float2 sx = make_float2(0.f, 0.f), sy = sx, sz = sx;
#pragma unroll UNROLL
    for (int q = q0; q < np; q += qs) {
        float2 dx, dy, dz;
        tx.sep(s, q, dx, dy, dz);
        const float4 b = s.B[q], d = s.D[q], e = s.E[q], xa = auxA[q], xb = auxB[q];
        const float2 inv = inv_r_x2_nz(dx, dy, dz, e2);
        const float2 mj = make_float2(b.z, b.w);
        const float2 vjx = make_float2(e.x, e.y), vjy = make_float2(e.z, e.w), vjz = make_float2(d.z, d.w);
        const float2 Ajx = make_float2(xa.x, xa.y), Ajy = make_float2(xa.z, xa.w), Ajz = make_float2(xb.x, xb.y);
        const float2 dvj = __ffma2_rn(dx, vjx, __ffma2_rn(dy, vjy, __fmul2_rn(dz, vjz)));
        const float2 dvi4 = __ffma2_rn(dx, n4x, __ffma2_rn(dy, n4y, __fmul2_rn(dz, n4z)));  // -4 d.v_i
        const float2 nvj = __fmul2_rn(dvj, inv);
        float2 B = __fadd2_rn(Ki, make_float2(xb.z, xb.w));
        B = __ffma2_rn(n4x, vjx, B);
        B = __ffma2_rn(n4y, vjy, B);
        B = __ffma2_rn(n4z, vjz, B);
        B = __ffma2_rn(dx, Ajx, B);
        B = __ffma2_rn(dy, Ajy, B);
        B = __ffma2_rn(dz, Ajz, B);
        B = __ffma2_rn(__fmul2_rn(nvj, nvj), make_float2(-1.5f, -1.5f), B);
        const float2 Wr = __ffma2_rn(dvj, make_float2(3.f, 3.f), dvi4);  // W r
        const float2 ms = __fmul2_rn(mj, inv);
        const float2 k3 = __fmul2_rn(ms, __fmul2_rn(inv, inv));
        const float2 fb = __fmul2_rn(k3, B), fW = __fmul2_rn(k3, Wr);
        const float2 g7 = __fmul2_rn(ms, make_float2(7.f, 7.f));
        sx = __ffma2_rn(g7, Ajx, __ffma2_rn(fW, __ffma2_rn(vjx, m1, vix), __ffma2_rn(fb, dx, sx)));
        sy = __ffma2_rn(g7, Ajy, __ffma2_rn(fW, __ffma2_rn(vjy, m1, viy), __ffma2_rn(fb, dy, sy)));
        sz = __ffma2_rn(g7, Ajz, __ffma2_rn(fW, __ffma2_rn(vjz, m1, viz), __ffma2_rn(fb, dz, sz)));
    }
    S = make_float3(sx.x + sx.y, sy.x + sy.y, sz.x + sz.y);
}

// FP64: sources j = j0, j0 + js, ... < n; aux[j] = (A_j, Phi_j).
template <int UNROLL>
__device__ __forceinline__ void eih_terms_f64(const EnsSlab<false>& s, const double4* __restrict__ aux, int n,
                                              int j0, int js, double4 xi, double4 vi, double4 ai, double eps2,
                                              double3& S) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll UNROLL
    for (int j = j0; j < n; j += js) {
        const double4 xj = s.x[j], vj = s.v[j], aj = aux[j];
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double d2 = fma(dx, dx, fma(dy, dy, dz * dz));
        const double inv = d2 > 0.0 ? rsqrt(d2 + eps2) : 0.0;  // not the target itself
        const double inv2 = inv * inv;
        const double vij = vi.x * vj.x + vi.y * vj.y + vi.z * vj.z;
        const double dvi = dx * vi.x + dy * vi.y + dz * vi.z;
        const double dvj = dx * vj.x + dy * vj.y + dz * vj.z;
        const double dA = dx * aj.x + dy * aj.y + dz * aj.z;
        const double nvj = dvj * inv;
        const double B = -4.0 * ai.w - aj.w + vi.w + 2.0 * vj.w - 4.0 * vij - 1.5 * nvj * nvj + 0.5 * dA;
        const double W = (3.0 * dvj - 4.0 * dvi) * inv;
        const double f = xj.w * inv2, fb = f * inv * B, g7 = 3.5 * xj.w * inv;
        sx += fb * dx + f * W * (vi.x - vj.x) + g7 * aj.x;
        sy += fb * dy + f * W * (vi.y - vj.y) + g7 * aj.y;
        sz += fb * dz + f * W * (vi.z - vj.z) + g7 * aj.z;
    }
    S = make_double3(sx, sy, sz);
}

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
// MIXED, with aux pair-interleaved like the slab: 32 float4 of
// (A_x, A_x', A_y, A_y') / 2 then 32 of (A_z / 2, A_z' / 2, Q, Q'),
// Q = 2 |v|^2 - Phi).
template <bool MIXED, int UNROLL>
__device__ __forceinline__ void eih_accel(const EnsSlab<MIXED>& slab, typename EnsAux<MIXED>::T4* aux, int n,
                                          int lane, bool two, bool v0, bool v1, bool sec, int sb, int sub, int lps,
                                          double eps2, double G, double c2, double a[2][3]) {
    const int np = (n + 1) >> 1;
    double A[2][4];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (q == 1 && !two) { A[1][0] = A[1][1] = A[1][2] = A[1][3] = 0.0; continue; }
        const int idx = q ? (sec ? 32 + sb : 0) : (v0 ? lane : 0);
        double sx, sy, sz, sp;
        if constexpr (MIXED) {
            float3 aN;
            float ph;
            newton_phi_f32<UNROLL>(slab, np, q ? sub : 0, q ? lps : 1, slab_body(slab, idx), (float)eps2, aN, ph);
            sx = aN.x; sy = aN.y; sz = aN.z; sp = ph;
        } else {
            double3 aN;
            newton_phi_f64<UNROLL>(slab, n, q ? sub : 0, q ? lps : 1, slab.x[idx], eps2, aN, sp);
            sx = aN.x; sy = aN.y; sz = aN.z;
        }
        if (q == 1) {
            sx = group_total(sx, lps, lane, v1); sy = group_total(sy, lps, lane, v1);
            sz = group_total(sz, lps, lane, v1); sp = group_total(sp, lps, lane, v1);
        }
        const bool valid = q ? v1 : v0;  // zeros past n: a half-used last pair adds nothing
        A[q][0] = valid ? G * sx : 0.0; A[q][1] = valid ? G * sy : 0.0;
        A[q][2] = valid ? G * sz : 0.0; A[q][3] = valid ? G * sp : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (q == 1 && !two) continue;
        const int b = lane + 32 * q;
        if constexpr (MIXED) {  // A / 2 and Q = 2 |v|^2 - Phi, the forms eih_terms_f32 reads
            float* xa = reinterpret_cast<float*>(aux);
            float* xb = reinterpret_cast<float*>(aux + 32);
            const int o = pslot(b);
            const double w = (double)reinterpret_cast<const float*>(slab.F)[b];
            xa[o] = (float)(0.5 * A[q][0]); xa[o + 2] = (float)(0.5 * A[q][1]);
            xb[o] = (float)(0.5 * A[q][2]); xb[o + 2] = (float)(2.0 * w - A[q][3]);
        } else {
            if (q ? v1 : v0) aux[b] = make_double4(A[q][0], A[q][1], A[q][2], A[q][3]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (q == 1 && !two) { a[1][0] = a[1][1] = a[1][2] = 0.0; continue; }
        const int idx = q ? (sec ? 32 + sb : 0) : (v0 ? lane : 0);
        double sx, sy, sz;
        if constexpr (MIXED) {
            const float4* xa = reinterpret_cast<const float4*>(aux);
            const float Q_i = reinterpret_cast<const float*>(aux + 32)[pslot(idx) + 2];
            float3 S;
            eih_terms_f32<UNROLL>(slab, xa, xa + 32, np, q ? sub : 0, q ? lps : 1, slab_body(slab, idx), Q_i,
                                  (float)eps2, S);
            sx = S.x; sy = S.y; sz = S.z;
        } else {
            double3 S;
            eih_terms_f64<UNROLL>(slab, aux, n, q ? sub : 0, q ? lps : 1, slab.x[idx], slab.v[idx], aux[idx], eps2,
                                  S);
            sx = S.x; sy = S.y; sz = S.z;
        }
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
        const int sys = order ? order[w] : (int)w;  // no order: upload order
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
                    const int idx = lane + 32 * q;
                    if constexpr (MIXED) {
                        // every slot the pairs can reach: lanes past n hold zero state
                        if (q == 1 && !two) continue;
                        slab_put(slab, idx, x[q], v[q]);
                    } else {
                        if (!(q ? v1 : v0)) continue;
                        const double vsq = v[q].x * v[q].x + v[q].y * v[q].y + v[q].z * v[q].z;
                        slab.x[idx] = x[q];
                        slab.v[idx] = make_double4(v[q].x, v[q].y, v[q].z, vsq);
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
                    double sx, sy, sz;
                    if constexpr (MIXED) {
                        // source pairs, split among the lps lanes for q = 1
                        float3 aN, a1, a2;
                        accel_f32<PNL, UNROLL>(slab, (n + 1) >> 1, q ? sub : 0, q ? lps : 1, slab_body(slab, idx),
                                               epsf, Gf, pkf, aN, a1, a2);
                        sx = ((double)aN.x + (double)a1.x) + (double)a2.x;
                        sy = ((double)aN.y + (double)a1.y) + (double)a2.y;
                        sz = ((double)aN.z + (double)a1.z) + (double)a2.z;
                    } else {
                        accel_f64<PNL, UNROLL>(slab, n, q ? sub : 0, q ? lps : 1, slab.x[idx], slab.v[idx], eps2, G,
                                               pk, sx, sy, sz);
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
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 > 0.0) phi += G * xj.w / sqrt(d2 + eps2);
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
                    bool use_graph, bool lpt) {
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
        kern<<<(unsigned)blocks, wpb * 32, smem, s>>>(e.nsys, lpt ? e.order.as<int32_t>() : nullptr, e.off.as<int32_t>(),
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
                    int check_every, bool g, bool lpt) {
    switch (unroll) {
        case 1: return launch_ensemble<MIXED, PNL, 1>(c, p, k, nsteps, wpb, check_every, g, lpt);
        case 4: return launch_ensemble<MIXED, PNL, 4>(c, p, k, nsteps, wpb, check_every, g, lpt);
        default: return launch_ensemble<MIXED, PNL, 2>(c, p, k, nsteps, wpb, check_every, g, lpt);
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
    const int schedule = cfg ? cfg->schedule : 0;
    if (wpb < 1 || wpb > 16 || (unroll != 1 && unroll != 2 && unroll != 4) || check < 1) return ASTER_ERR_INVALID_ARG;
    if (schedule != 0 && schedule != 1) return ASTER_ERR_INVALID_ARG;
    const bool lpt = schedule == 0;
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    *c->ens.cancel_host = 0;
    const Coeffs k = make_coeffs(integrator, p->dt);
    // PN level: 3 EIH; 2 when a 2PN or 2.5PN term is requested, else 1 for 1PN alone
    cudaEventRecord(c->ev[0], c->stream);
    int st;
    if (precision == ASTER_MIXED)
        st = pnl == 3 ? dispatch_unroll<true, 3>(c, p, k, nsteps, wpb, unroll, check, graph, lpt)
           : pnl == 2 ? dispatch_unroll<true, 2>(c, p, k, nsteps, wpb, unroll, check, graph, lpt)
           : pnl == 1 ? dispatch_unroll<true, 1>(c, p, k, nsteps, wpb, unroll, check, graph, lpt)
                      : dispatch_unroll<true, 0>(c, p, k, nsteps, wpb, unroll, check, graph, lpt);
    else
        st = pnl == 3 ? dispatch_unroll<false, 3>(c, p, k, nsteps, wpb, unroll, check, graph, lpt)
           : pnl == 2 ? dispatch_unroll<false, 2>(c, p, k, nsteps, wpb, unroll, check, graph, lpt)
           : pnl == 1 ? dispatch_unroll<false, 1>(c, p, k, nsteps, wpb, unroll, check, graph, lpt)
                      : dispatch_unroll<false, 0>(c, p, k, nsteps, wpb, unroll, check, graph, lpt);
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
