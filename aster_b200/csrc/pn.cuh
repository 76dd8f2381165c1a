// Pairwise post-Newtonian terms of the reference's compute_gravitational
// (src/physics/tool_chain_impl.cpp:120-137): get_pn1 (c^-2, :110-118), get_pn2
// (c^-4, :79-107) and get_pn25 (c^-5, :65-77), selected by the force-law bits.
// Shared by the all-pairs kernels and the batched ensemble kernel.
#pragma once

#include "aster_internal.cuh"

// Post-Newtonian constants and the terms in use: f bit 0 = 1PN, bit 1 = 2PN,
// bit 2 = 2.5PN. PN level PNL (a template parameter of the kernels): 0 Newton
// only, 1 Newton + 1PN, 2 Newton + the terms f selects. c2 = c^-2, c4 = c^-4,
// ic = c^-1 (c^-5 is formed as c^-4 ic inside a product that stays in FP32
// range: c^-5 itself is below FP32's normal range in SI units).
template <class T>
struct PnK {
    T c2, c4, ic;
    int f;
};

// Acceleration on body i from body j, divided by G. j == i contributes 0 (zero
// separation and relative velocity). With n the unit vector from j to i (the
// reference's -norm), p_i = G m_i / r, p_j = G m_j / r:
//   1PN : c^-2 m_j/r^2 [n A + (v_i - v_j) B]
//   2PN : c^-4 m_j/r^2 [n S_n + (v_i - v_j) S_v + n (-57/4 p_i^2 - 9 p_j^2 - 69/2 p_i p_j)]
//   2.5PN: c^-5 4/5 p_i m_j/r^2 [(v_i - v_j) I_1 + n (n.(v_i - v_j)) I_2]
// with A, B, S_n, S_v, I_1, I_2 the scalar brackets of get_pn1, get_pn2 and
// get_pn25. The 2PN mass term is the reference's G^2 m_j/r^4 (-57/4 m_i^2 -
// 9 m_j^2 - 69/2 m_i m_j) written with p_i, p_j, which keeps every factor in
// FP32 range for masses of ~1e30 (m^2 would overflow).
template <class T>
struct PnPair {
    // per-pair inputs
    T nx, ny, nz, dvx, dvy, dvz, inv, inv2, mi, mj, vi2, vj2, v12, nv1, nv2, G;
    __device__ __forceinline__ void pn1(T c2, T& px, T& py, T& pz) const {
        const T A = -vi2 - T(2) * vj2 + T(4) * v12 + T(1.5) * nv2 * nv2 + (T(5) * mi + T(4) * mj) * G * inv;
        const T B = T(4) * nv1 - T(3) * nv2;
        const T f = mj * inv2 * c2;
        px += (nx * A + dvx * B) * f;
        py += (ny * A + dvy * B) * f;
        pz += (nz * A + dvz * B) * f;
    }
    __device__ __forceinline__ void pn2(T c4, T& qx, T& qy, T& qz) const {
        const T nv22 = nv2 * nv2, nv12 = nv1 * nv1;
        const T p1 = G * mi * inv, p2 = G * mj * inv;
        const T Sn = T(-2) * vj2 * vj2 + T(4) * vj2 * v12 - T(2) * v12 * v12 + T(1.5) * vi2 * nv22 +
                     T(4.5) * vj2 * nv22 - T(6) * v12 * nv22 - T(1.875) * nv22 * nv22 +
                     p1 * (T(-3.75) * vi2 + T(1.25) * vj2 - T(2.5) * v12 + T(19.5) * nv12 - T(39) * nv1 * nv2 +
                           T(8.5) * nv22) +
                     p2 * (T(4) * vj2 - T(8) * v12 + T(2) * nv12 - T(4) * nv1 * nv2 - T(6) * nv22);
        const T Sv = vi2 * nv2 + T(4) * vj2 * nv1 - T(5) * vj2 * nv2 - T(4) * v12 * nv1 + T(4) * v12 * nv2 -
                     T(6) * nv1 * nv22 + T(4.5) * nv22 * nv2 + p1 * (T(-15.75) * nv1 + T(13.75) * nv2) +
                     p2 * (T(-2) * nv1 - T(2) * nv2);
        const T Sm = T(-14.25) * p1 * p1 - T(9) * p2 * p2 - T(34.5) * p1 * p2;
        const T f = mj * inv2 * c4;
        qx += f * (nx * (Sn + Sm) + dvx * Sv);
        qy += f * (ny * (Sn + Sm) + dvy * Sv);
        qz += f * (nz * (Sn + Sm) + dvz * Sv);
    }
    __device__ __forceinline__ void pn25(T c4, T ic, T& qx, T& qy, T& qz) const {
        const T p1 = G * mi * inv, p2 = G * mj * inv;
        const T sq = dvx * dvx + dvy * dvy + dvz * dvz;
        const T I1 = -sq + T(2) * p1 - T(8) * p2;
        const T I2 = (nv1 - nv2) * (T(3) * sq - T(6) * p1 + T(52) / T(3) * p2);
        const T f = T(0.8) * p1 * (mj * inv2 * c4) * ic;
        qx += (dvx * I1 + nx * I2) * f;
        qy += (dvy * I1 + ny * I2) * f;
        qz += (dvz * I1 + nz * I2) * f;
    }
};

// Newton + 1PN for two sources at once with the paired FP32 instructions of
// sm_100 (add/mul/fma .f32x2), one source in each half of every operand.
// d = x_j - x_i (both sources), mj their masses, vj their velocities and
// vj2 = |v_j|^2; per target, broadcast to both halves: vi its velocity,
// vi4 = 4 v_i, nvi2 = -|v_i|^2 and mi5G = 5 G m_i; G4 = 4 G. Adds the
// Newtonian m_j d / r^3 to a (divided by G) and to p the 1PN sum
//   P = sum_j m_j r^-3 [d A + (v_i - v_j) B'],
//   A = -|v_i|^2 - 2 |v_j|^2 + 4 v_i.v_j + 3/2 (d.v_j / r)^2 + (5 m_i + 4 m_j) G / r,
//   B' = 4 d.v_i - 3 d.v_j,
// whose -c^-2 multiple is the 1PN acceleration divided by G: PnPair::pn1 with
// n = -d / r, B = -B' / r and f = c^-2 m_j / r^2 gathered into m_j r^-3, so
// that the unit vector and f cost no instructions of their own. GUARD: a zero
// r^2 (the target itself when unsoftened) contributes nothing.
template <bool GUARD>
__device__ __forceinline__ void newton_pn1_x2(const float2 dx, const float2 dy, const float2 dz, const float2 mj,
                                              const float2 vjx, const float2 vjy, const float2 vjz, const float2 vj2,
                                              const float2 vix, const float2 viy, const float2 viz,
                                              const float2 vi4x, const float2 vi4y, const float2 vi4z,
                                              const float2 nvi2, const float2 mi5G, const float2 eps2,
                                              const float2 G4, float2& ax, float2& ay, float2& az, float2& px,
                                              float2& py, float2& pz) {
    float2 r2 = __ffma2_rn(dz, dz, eps2);
    r2 = __ffma2_rn(dy, dy, r2);
    r2 = __ffma2_rn(dx, dx, r2);
    float2 s = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    if (GUARD) {
        s.x = r2.x > 0.f ? s.x : 0.f;
        s.y = r2.y > 0.f ? s.y : 0.f;
    }
    const float2 ms = __fmul2_rn(mj, s);
    const float2 sN = __fmul2_rn(ms, __fmul2_rn(s, s));  // m_j / r^3
    ax = __ffma2_rn(dx, sN, ax);
    ay = __ffma2_rn(dy, sN, ay);
    az = __ffma2_rn(dz, sN, az);
    const float2 w = __ffma2_rn(dx, vjx, __ffma2_rn(dy, vjy, __fmul2_rn(dz, vjz)));     // d.v_j
    const float2 u4 = __ffma2_rn(dx, vi4x, __ffma2_rn(dy, vi4y, __fmul2_rn(dz, vi4z)));  // 4 d.v_i
    const float2 Bp = __ffma2_rn(w, make_float2(-3.f, -3.f), u4);
    const float2 ws = __fmul2_rn(w, s);
    float2 A = __ffma2_rn(vj2, make_float2(-2.f, -2.f), nvi2);
    A = __ffma2_rn(vi4x, vjx, A);
    A = __ffma2_rn(vi4y, vjy, A);
    A = __ffma2_rn(vi4z, vjz, A);
    A = __ffma2_rn(__fmul2_rn(ws, ws), make_float2(1.5f, 1.5f), A);
    A = __ffma2_rn(ms, G4, A);
    A = __ffma2_rn(s, mi5G, A);
    const float2 sA = __fmul2_rn(sN, A), sB = __fmul2_rn(sN, Bp);
    const float2 m1 = make_float2(-1.f, -1.f);
    const float2 dvx = __ffma2_rn(vjx, m1, vix), dvy = __ffma2_rn(vjy, m1, viy), dvz = __ffma2_rn(vjz, m1, viz);
    px = __ffma2_rn(dx, sA, __ffma2_rn(dvx, sB, px));
    py = __ffma2_rn(dy, sA, __ffma2_rn(dvy, sB, py));
    pz = __ffma2_rn(dz, sA, __ffma2_rn(dvz, sB, pz));
}

// Newton and every post-Newtonian term the flags select (bit 0 1PN, bit 1 2PN,
// bit 2 2.5PN), two sources per paired FP32 instruction: the algebra of
// PnPair::pn1/pn2/pn25 with the sums gathered under the Newtonian factor
// m_j / r^3 and the c^-2, c^-4 factors applied once per target, as in
// newton_pn1_x2. Inputs as newton_pn1_x2's, plus vi2 = |v_i|^2 and
// Gmi = G m_i per target and nk = -0.8 c^-1. Adds m_j d / r^3 to a, to p the
// 1PN sum P of newton_pn1_x2 (the 1PN term is -c^-2 P) and to q the sum Q whose
// -c^-4 multiple is the 2PN + 2.5PN term (all divided by G). With
// n = -d s, nv1 = n.v_i = -s d.v_i, nv2 = -s d.v_j, p1 = G m_i s, p2 = G m_j s:
//   2PN:   c^-4 m_j s^2 [n (Sn + Sm) + dv Sv] = -c^-4 [m_j s^3 (Sn + Sm) d - m_j s^2 Sv dv],
//   2.5PN: 0.8 c^-5 p1 m_j s^2 [dv I1 + n I2] = -c^-4 (-0.8 c^-1) p1 m_j s^2 [dv I1 - s I2 d].
template <bool GUARD>
__device__ __forceinline__ void newton_pn_all_x2(const float2 dx, const float2 dy, const float2 dz, const float2 mj,
                                                 const float2 vjx, const float2 vjy, const float2 vjz,
                                                 const float2 vj2, const float2 vix, const float2 viy,
                                                 const float2 viz, const float2 vi4x, const float2 vi4y,
                                                 const float2 vi4z, const float2 nvi2, const float2 vi2,
                                                 const float2 mi5G, const float2 Gmi, const float2 eps2,
                                                 const float2 G4, const float2 G2, const float2 nk, int f,
                                                 float2& ax, float2& ay, float2& az, float2& px, float2& py,
                                                 float2& pz, float2& qx, float2& qy, float2& qz) {
    auto k2 = [](float v) { return make_float2(v, v); };
    float2 r2 = __ffma2_rn(dz, dz, eps2);
    r2 = __ffma2_rn(dy, dy, r2);
    r2 = __ffma2_rn(dx, dx, r2);
    float2 s = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    if (GUARD) {
        s.x = r2.x > 0.f ? s.x : 0.f;
        s.y = r2.y > 0.f ? s.y : 0.f;
    }
    const float2 ms = __fmul2_rn(mj, s);
    const float2 mss = __fmul2_rn(ms, s);   // m_j / r^2
    const float2 sN = __fmul2_rn(mss, s);   // m_j / r^3
    ax = __ffma2_rn(dx, sN, ax);
    ay = __ffma2_rn(dy, sN, ay);
    az = __ffma2_rn(dz, sN, az);
    if (!(f & 7)) return;
    const float2 m1 = k2(-1.f);
    const float2 w = __ffma2_rn(dx, vjx, __ffma2_rn(dy, vjy, __fmul2_rn(dz, vjz)));     // d.v_j
    const float2 u4 = __ffma2_rn(dx, vi4x, __ffma2_rn(dy, vi4y, __fmul2_rn(dz, vi4z)));  // 4 d.v_i
    const float2 dvx = __ffma2_rn(vjx, m1, vix), dvy = __ffma2_rn(vjy, m1, viy), dvz = __ffma2_rn(vjz, m1, viz);
    if (f & 1) {  // 1PN: newton_pn1_x2's sum
        const float2 Bp = __ffma2_rn(w, k2(-3.f), u4);
        const float2 ws = __fmul2_rn(w, s);
        float2 A = __ffma2_rn(vj2, k2(-2.f), nvi2);
        A = __ffma2_rn(vi4x, vjx, A);
        A = __ffma2_rn(vi4y, vjy, A);
        A = __ffma2_rn(vi4z, vjz, A);
        A = __ffma2_rn(__fmul2_rn(ws, ws), k2(1.5f), A);
        A = __ffma2_rn(ms, G4, A);
        A = __ffma2_rn(s, mi5G, A);
        const float2 sA = __fmul2_rn(sN, A), sB = __fmul2_rn(sN, Bp);
        px = __ffma2_rn(dx, sA, __ffma2_rn(dvx, sB, px));
        py = __ffma2_rn(dy, sA, __ffma2_rn(dvy, sB, py));
        pz = __ffma2_rn(dz, sA, __ffma2_rn(dvz, sB, pz));
    }
    if (!(f & 6)) return;
    const float2 nv1 = __fmul2_rn(u4, __fmul2_rn(s, k2(-0.25f)));  // n.v_i
    const float2 nv2 = __fmul2_rn(__fmul2_rn(w, s), m1);           // n.v_j
    const float2 v12 = __ffma2_rn(vix, vjx, __ffma2_rn(viy, vjy, __fmul2_rn(viz, vjz)));
    const float2 p1 = __fmul2_rn(Gmi, s), p2 = __fmul2_rn(G2, ms);  // G m_i / r, G m_j / r
    if (f & 2) {  // 2PN (PnPair::pn2)
        const float2 nv22 = __fmul2_rn(nv2, nv2), nv12 = __fmul2_rn(nv1, nv1), n12 = __fmul2_rn(nv1, nv2);
        // -2 vj2^2 + 4 vj2 v12 - 2 v12^2 = -2 (vj2 - v12)^2
        const float2 t = __ffma2_rn(v12, m1, vj2);
        float2 Sn = __fmul2_rn(__fmul2_rn(t, t), k2(-2.f));
        // + nv22 (1.5 vi2 + 4.5 vj2 - 6 v12) - 1.875 nv22^2
        const float2 c1 = __ffma2_rn(v12, k2(-6.f), __ffma2_rn(vj2, k2(4.5f), __fmul2_rn(vi2, k2(1.5f))));
        Sn = __ffma2_rn(nv22, c1, Sn);
        Sn = __ffma2_rn(__fmul2_rn(nv22, nv22), k2(-1.875f), Sn);
        // + p1 (-3.75 vi2 + 1.25 vj2 - 2.5 v12 + 19.5 nv12 - 39 nv1 nv2 + 8.5 nv22)
        float2 e1 = __ffma2_rn(vj2, k2(1.25f), __fmul2_rn(vi2, k2(-3.75f)));
        e1 = __ffma2_rn(v12, k2(-2.5f), e1);
        e1 = __ffma2_rn(nv12, k2(19.5f), e1);
        e1 = __ffma2_rn(n12, k2(-39.f), e1);
        e1 = __ffma2_rn(nv22, k2(8.5f), e1);
        Sn = __ffma2_rn(p1, e1, Sn);
        // + p2 (4 vj2 - 8 v12 + 2 nv12 - 4 nv1 nv2 - 6 nv22)
        float2 e2 = __ffma2_rn(v12, k2(-8.f), __fmul2_rn(vj2, k2(4.f)));
        e2 = __ffma2_rn(nv12, k2(2.f), e2);
        e2 = __ffma2_rn(n12, k2(-4.f), e2);
        e2 = __ffma2_rn(nv22, k2(-6.f), e2);
        Sn = __ffma2_rn(p2, e2, Sn);
        // Sv = nv1 (4 vj2 - 4 v12 - 6 nv22 - 15.75 p1 - 2 p2) + nv2 (vi2 - 5 vj2 + 4 v12 + 4.5 nv22 + 13.75 p1 - 2 p2)
        float2 A1 = __ffma2_rn(v12, k2(-4.f), __fmul2_rn(vj2, k2(4.f)));
        A1 = __ffma2_rn(nv22, k2(-6.f), A1);
        A1 = __ffma2_rn(p1, k2(-15.75f), A1);
        A1 = __ffma2_rn(p2, k2(-2.f), A1);
        float2 A2 = __ffma2_rn(vj2, k2(-5.f), vi2);
        A2 = __ffma2_rn(v12, k2(4.f), A2);
        A2 = __ffma2_rn(nv22, k2(4.5f), A2);
        A2 = __ffma2_rn(p1, k2(13.75f), A2);
        A2 = __ffma2_rn(p2, k2(-2.f), A2);
        const float2 Sv = __ffma2_rn(nv1, A1, __fmul2_rn(nv2, A2));
        // Sm = -14.25 p1^2 - 9 p2^2 - 34.5 p1 p2
        const float2 Sm = __ffma2_rn(p1, __ffma2_rn(p1, k2(-14.25f), __fmul2_rn(p2, k2(-34.5f))),
                                     __fmul2_rn(__fmul2_rn(p2, p2), k2(-9.f)));
        // Q += m_j s^3 (Sn + Sm) d - m_j s^2 Sv dv
        const float2 a1 = __fmul2_rn(sN, __fadd2_rn(Sn, Sm)), a2 = __fmul2_rn(__fmul2_rn(mss, Sv), m1);
        qx = __ffma2_rn(dx, a1, __ffma2_rn(dvx, a2, qx));
        qy = __ffma2_rn(dy, a1, __ffma2_rn(dvy, a2, qy));
        qz = __ffma2_rn(dz, a1, __ffma2_rn(dvz, a2, qz));
    }
    if (f & 4) {  // 2.5PN (PnPair::pn25)
        const float2 sq = __ffma2_rn(dvx, dvx, __ffma2_rn(dvy, dvy, __fmul2_rn(dvz, dvz)));
        const float2 I1 = __ffma2_rn(p2, k2(-8.f), __ffma2_rn(p1, k2(2.f), __fmul2_rn(sq, m1)));
        const float2 I2 = __fmul2_rn(__fadd2_rn(nv1, __fmul2_rn(nv2, m1)),
                                     __ffma2_rn(p2, k2(52.f / 3.f), __ffma2_rn(sq, k2(3.f), __fmul2_rn(p1, k2(-6.f)))));
        // Q += (-0.8 c^-1) p1 m_j s^2 (dv I1 - s I2 d)
        const float2 g = __fmul2_rn(__fmul2_rn(p1, mss), nk);
        const float2 gI1 = __fmul2_rn(g, I1), gsI2 = __fmul2_rn(__fmul2_rn(g, s), __fmul2_rn(I2, m1));
        qx = __ffma2_rn(dvx, gI1, __ffma2_rn(dx, gsI2, qx));
        qy = __ffma2_rn(dvy, gI1, __ffma2_rn(dy, gsI2, qy));
        qz = __ffma2_rn(dvz, gI1, __ffma2_rn(dz, gsI2, qz));
    }
}

// The terms of level PNL: 1PN into p, 2PN and 2.5PN into q (kept apart in
// FP32 so that the smaller corrections are not lost against the larger sums).
template <int PNL, class T>
__device__ __forceinline__ void pn_terms(const PnK<T>& k, const PnPair<T>& q, T& px, T& py, T& pz, T& qx, T& qy,
                                         T& qz) {
    if (PNL == 1 || (PNL == 2 && (k.f & 1))) q.pn1(k.c2, px, py, pz);
    if (PNL == 2 && (k.f & 2)) q.pn2(k.c4, qx, qy, qz);
    if (PNL == 2 && (k.f & 4)) q.pn25(k.c4, k.ic, qx, qy, qz);
}

// The force-law bits of p as PN constants (powers of 1/c formed in the
// reference's order, inv_c * inv_c * ...).
inline PnK<double> make_pn(const aster_params* p) {
    PnK<double> k{0.0, 0.0, 0.0, 0};
    k.f = ((p->force_law & ASTER_PN1) ? 1 : 0) | ((p->force_law & ASTER_PN2) ? 2 : 0) |
          ((p->force_law & ASTER_PN25) ? 4 : 0);
    if (k.f) {
        const double ic = 1.0 / p->c;
        k.c2 = ic * ic;
        k.c4 = ic * ic * ic * ic;
        k.ic = ic;
    }
    return k;
}

// PN level of a force law: 0, 1 (1PN only) or 2 (2PN or 2.5PN present).
inline int pn_level(const aster_params* p) {
    if (p->force_law & (ASTER_PN2 | ASTER_PN25)) return 2;
    return (p->force_law & ASTER_PN1) ? 1 : 0;
}

__host__ __device__ inline PnK<float> pn_float(const PnK<double>& k) { return PnK<float>{(float)k.c2, (float)k.c4, (float)k.ic, k.f}; }
