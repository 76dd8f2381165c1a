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
