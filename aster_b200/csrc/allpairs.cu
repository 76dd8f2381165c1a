// All-pairs force kernels: the replacement for Parallelized::compute_forces
// (src/utils/builder_endpoint.cpp:729-757), SimpleGPU::compute_forces +
// cl3d_newton (src/solvers/SimpleGPU.cpp:17-71,
// include/Aster/kernels/newton_update3d.cl.h:28-72) and the pair law of
// compute_gravitational (src/physics/tool_chain_impl.cpp:120-137) with every
// post-Newtonian term it offers (get_pn1, get_pn2, get_pn25; pn.cuh).
//
// Pair law (acceleration on i from j, d = x_j - x_i, r^2 = d.d + eps2):
//   a_i += G m_j d / r^3
//   PN1:  + G m_j / (c^2 r^2) [ n A + (v_i - v_j) B ],  n = -d/r,
//         A = -v_i^2 - 2 v_j^2 + 4 v_i.v_j + 1.5 (n.v_j)^2 + 5 G m_i/r + 4 G m_j/r,
//         B = 4 n.v_i - 3 n.v_j                  (tool_chain_impl.cpp:110-118)
//   PN2, PN2.5: the c^-4 and c^-5 terms (tool_chain_impl.cpp:65-107)
//
// Two arithmetic paths, one tiling:
//  * FP64: double4 (x,y,z,m) j-tiles in shared memory, FP64 throughout; the
//    "plain FP64 GPU path" the mixed path is measured against.
//  * MIXED: positions as double-single float pairs (hi = rn(x), lo = rn(x-hi)),
//    d = (x_j,hi - x_i,hi) + (x_j,lo - x_i,lo) in FP32 (accurate to FP32
//    relative precision of d even for close pairs far from the origin),
//    rsqrt on the SFU, per-thread FP32 partial sums over 64 j folded into a
//    two-sum compensated accumulator (hi, lo), final value in FP64.
// Each thread owns IPT targets; a block of BLOCK threads owns BLOCK*IPT targets
// and walks one j-slice; small n use several j-slices whose partial sums are
// added by k_reduce_slices (scratch memory).
#include "aster_internal.cuh"
#include "pn.cuh"

namespace {

constexpr int BLOCK = 128;   // threads per block == j-tile length
constexpr int IPT = 2;       // targets per thread
constexpr int FOLD = 64;     // FP32 terms summed before a compensated fold
constexpr float PAD_POS = 1.0e30f;

struct KickArgs {
    bool on;
    double half_dt;
    double4* vel;
};

// Epilogue shared by both paths: write acceleration (scaled by G) either to
// ctx->acc (+ optional closing kick v += a dt/2) or to an explicit output, or
// as a partial sum of slice s to scratch.
__device__ __forceinline__ void store_result(int64_t t, int64_t body, double ax, double ay, double az,
                                             double G, int nslices, int slice, int64_t nt,
                                             double4* __restrict__ partial, double4* __restrict__ acc,
                                             double* __restrict__ out3, KickArgs kick) {
    if (nslices > 1) {
        partial[(int64_t)slice * nt + t] = make_double4(ax, ay, az, 0.0);
        return;
    }
    ax *= G; ay *= G; az *= G;
    if (out3) {
        out3[3 * t] = ax; out3[3 * t + 1] = ay; out3[3 * t + 2] = az;
        return;
    }
    acc[body] = make_double4(ax, ay, az, 0.0);
    if (kick.on) {
        double4 v = kick.vel[body];
        v.x += ax * kick.half_dt; v.y += ay * kick.half_dt; v.z += az * kick.half_dt;
        kick.vel[body] = v;
    }
}

// ---------------------------------------------------------------- FP64 path
// PNL: 0 Newton, 1 Newton + 1PN, 2 Newton + the PN terms pk.f selects.
template <int PNL, bool GUARD>
__global__ void __launch_bounds__(BLOCK) k_allpairs_fp64(
    int64_t j_lo, int64_t n, int64_t nt, const int32_t* __restrict__ targets, const double4* __restrict__ pm,
    const double4* __restrict__ vel, double G, double eps2, PnK<double> pk, int64_t slice_len, int nslices,
    double4* __restrict__ partial, double4* __restrict__ acc, double* __restrict__ out3, KickArgs kick) {
    __shared__ double4 sp[BLOCK];
    __shared__ double4 sv[PNL ? BLOCK : 1];  // (vx, vy, vz, |v|^2)
    const int slice = blockIdx.y;
    const int64_t j0 = j_lo + (int64_t)slice * slice_len;  // sources [j_lo, n), sliced
    const int64_t j1 = min(n, j0 + slice_len);
    int64_t tt[IPT], bi[IPT];
    double xi[IPT], yi[IPT], zi[IPT], mi[IPT], vxi[IPT], vyi[IPT], vzi[IPT], v1sq[IPT];
    double ax[IPT], ay[IPT], az[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        tt[k] = (int64_t)blockIdx.x * BLOCK * IPT + k * BLOCK + threadIdx.x;
        bi[k] = tt[k] < nt ? (targets ? (int64_t)targets[tt[k]] : tt[k]) : 0;
        double4 p = pm[bi[k]];
        xi[k] = p.x; yi[k] = p.y; zi[k] = p.z; mi[k] = p.w;
        if (PNL) {
            double4 v = vel[bi[k]];
            vxi[k] = v.x; vyi[k] = v.y; vzi[k] = v.z;
            v1sq[k] = v.x * v.x + v.y * v.y + v.z * v.z;
        }
        ax[k] = ay[k] = az[k] = 0.0;
    }
    for (int64_t base = j0; base < j1; base += BLOCK) {
        const int64_t j = base + threadIdx.x;
        __syncthreads();
        sp[threadIdx.x] = j < j1 ? pm[j] : make_double4(1e300, 1e300, 1e300, 0.0);
        if (PNL) {
            double4 v = j < j1 ? vel[j] : make_double4(0, 0, 0, 0);
            v.w = v.x * v.x + v.y * v.y + v.z * v.z;
            sv[threadIdx.x] = v;
        }
        __syncthreads();
        const int cnt = (int)min((int64_t)BLOCK, j1 - base);  // a partial last tile stops at its last source
#pragma unroll 8
        for (int q = 0; q < cnt; ++q) {
            const double4 pj = sp[q];
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                double dx = pj.x - xi[k], dy = pj.y - yi[k], dz = pj.z - zi[k];
                double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
                double inv = rsqrt(r2);
                if (GUARD) inv = r2 > 0.0 ? inv : 0.0;
                double inv2 = inv * inv;
                double s = pj.w * inv * inv2;
                ax[k] = fma(dx, s, ax[k]); ay[k] = fma(dy, s, ay[k]); az[k] = fma(dz, s, az[k]);
                if (PNL) {
                    const double4 vj = sv[q];
                    PnPair<double> w;
                    w.nx = -dx * inv; w.ny = -dy * inv; w.nz = -dz * inv;
                    w.dvx = vxi[k] - vj.x; w.dvy = vyi[k] - vj.y; w.dvz = vzi[k] - vj.z;
                    w.inv = inv; w.inv2 = inv2; w.mi = mi[k]; w.mj = pj.w; w.vi2 = v1sq[k]; w.vj2 = vj.w;
                    w.v12 = vxi[k] * vj.x + vyi[k] * vj.y + vzi[k] * vj.z;
                    w.nv1 = w.nx * vxi[k] + w.ny * vyi[k] + w.nz * vzi[k];
                    w.nv2 = w.nx * vj.x + w.ny * vj.y + w.nz * vj.z;
                    w.G = G;  // the sums are accelerations / G; G is applied in store_result
                    pn_terms<PNL>(pk, w, ax[k], ay[k], az[k], ax[k], ay[k], az[k]);
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k)
        if (tt[k] < nt) store_result(tt[k], bi[k], ax[k], ay[k], az[k], G, nslices, slice, nt, partial, acc, out3, kick);
}

// --------------------------------------------------------------- mixed path
// With post-Newtonian terms (PNL 1: Newton + 1PN; 2: the terms the force-law
// bits select), two sources per paired FP32 instruction as in the Newtonian
// kernel below, one target per thread: the j-tile staged pair-interleaved
// (double-single positions, masses, velocities and |v|^2, as the batched
// ensemble's slab), the pair terms of pn.cuh (newton_pn1_x2,
// newton_pn_all_x2); the Newtonian sum folded into compensated sums every
// FOLD sources, the 1PN and 2PN + 2.5PN sums kept apart in FP32.
constexpr int IPT_PN = 1;

template <int PNL, bool GUARD>
__global__ void __launch_bounds__(BLOCK) k_allpairs_mixed_pn(
    int64_t j_lo, int64_t n, int64_t nt, const int32_t* __restrict__ targets, const float4* __restrict__ phi,
    const float4* __restrict__ plo, const float4* __restrict__ vf, float G, float eps2, PnK<float> pk,
    double Gd, int64_t slice_len, int nslices, double4* __restrict__ partial, double4* __restrict__ acc,
    double* __restrict__ out3, KickArgs kick) {
    // (hx hx' hy hy') (hz hz' m m') (lx lx' ly ly') (lz lz' vz vz') (vx vx' vy vy') (|v|^2 |v'|^2)
    __shared__ float4 pa[BLOCK / 2], pb[BLOCK / 2], pc[BLOCK / 2], pd[BLOCK / 2], pe[BLOCK / 2];
    __shared__ float2 pf[BLOCK / 2];
    const int slice = blockIdx.y;
    const int64_t j0 = j_lo + (int64_t)slice * slice_len;  // sources [j_lo, n), sliced
    const int64_t j1 = min(n, j0 + slice_len);
    const int64_t tt = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
    const int64_t bi = tt < nt ? (targets ? (int64_t)targets[tt] : tt) : 0;
    const float4 h = phi[bi], l = plo[bi], v = vf[bi];
    const float2 nhx = make_float2(-h.x, -h.x), nhy = make_float2(-h.y, -h.y), nhz = make_float2(-h.z, -h.z);
    const float2 nlx = make_float2(-l.x, -l.x), nly = make_float2(-l.y, -l.y), nlz = make_float2(-l.z, -l.z);
    const float w2 = v.x * v.x + v.y * v.y + v.z * v.z;
    const float2 vix = make_float2(v.x, v.x), viy = make_float2(v.y, v.y), viz = make_float2(v.z, v.z);
    const float2 vi4x = make_float2(4.f * v.x, 4.f * v.x), vi4y = make_float2(4.f * v.y, 4.f * v.y),
                 vi4z = make_float2(4.f * v.z, 4.f * v.z);
    const float2 nvi2 = make_float2(-w2, -w2), vi2 = make_float2(w2, w2);
    const float2 mi5G = make_float2(5.f * G * h.w, 5.f * G * h.w), Gmi = make_float2(G * h.w, G * h.w);
    const float2 G4 = make_float2(4.f * G, 4.f * G), G2 = make_float2(G, G), e2 = make_float2(eps2, eps2);
    const float2 nk = make_float2(-0.8f * pk.ic, -0.8f * pk.ic);
    float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax, px = ax, py = ax, pz = ax, qx = ax, qy = ax, qz = ax;
    CompSum cx, cy, cz;
    float* fa = reinterpret_cast<float*>(pa);
    float* fb = reinterpret_cast<float*>(pb);
    float* fc = reinterpret_cast<float*>(pc);
    float* fd = reinterpret_cast<float*>(pd);
    float* fe = reinterpret_cast<float*>(pe);
    float* ff = reinterpret_cast<float*>(pf);
    const int o = ((threadIdx.x >> 1) << 2) | (threadIdx.x & 1);
    for (int64_t base = j0; base < j1; base += BLOCK) {
        const int64_t j = base + threadIdx.x;
        __syncthreads();
        float4 sh = make_float4(PAD_POS, PAD_POS, PAD_POS, 0.f), sl = make_float4(0.f, 0.f, 0.f, 0.f), sv = sl;
        if (j < j1) { sh = phi[j]; sl = plo[j]; sv = vf[j]; }
        fa[o] = sh.x; fa[o + 2] = sh.y;
        fb[o] = sh.z; fb[o + 2] = sh.w;
        fc[o] = sl.x; fc[o + 2] = sl.y;
        fd[o] = sl.z; fd[o + 2] = sv.z;
        fe[o] = sv.x; fe[o + 2] = sv.y;
        ff[threadIdx.x] = sv.x * sv.x + sv.y * sv.y + sv.z * sv.z;
        __syncthreads();
        // a partial last tile stops at its last source pair (padding: no mass)
        const int npair = (int)((min((int64_t)BLOCK, j1 - base) + 1) / 2);
#pragma unroll 1
        for (int c0 = 0; c0 < npair; c0 += FOLD / 2) {
#pragma unroll 2
            for (int q = c0; q < min(c0 + FOLD / 2, npair); ++q) {
                const float4 A = pa[q], B = pb[q], C = pc[q], D = pd[q], E = pe[q];
                const float2 dx = __fadd2_rn(__fadd2_rn(make_float2(A.x, A.y), nhx), __fadd2_rn(make_float2(C.x, C.y), nlx));
                const float2 dy = __fadd2_rn(__fadd2_rn(make_float2(A.z, A.w), nhy), __fadd2_rn(make_float2(C.z, C.w), nly));
                const float2 dz = __fadd2_rn(__fadd2_rn(make_float2(B.x, B.y), nhz), __fadd2_rn(make_float2(D.x, D.y), nlz));
                if constexpr (PNL == 1)
                    newton_pn1_x2<GUARD>(dx, dy, dz, make_float2(B.z, B.w), make_float2(E.x, E.y),
                                         make_float2(E.z, E.w), make_float2(D.z, D.w), pf[q], vix, viy, viz, vi4x,
                                         vi4y, vi4z, nvi2, mi5G, e2, G4, ax, ay, az, px, py, pz);
                else
                    newton_pn_all_x2<GUARD>(dx, dy, dz, make_float2(B.z, B.w), make_float2(E.x, E.y),
                                            make_float2(E.z, E.w), make_float2(D.z, D.w), pf[q], vix, viy, viz,
                                            vi4x, vi4y, vi4z, nvi2, vi2, mi5G, Gmi, e2, G4, G2, nk, pk.f, ax, ay, az,
                                            px, py, pz, qx, qy, qz);
            }
            cx.add(ax.x + ax.y); cy.add(ay.x + ay.y); cz.add(az.x + az.y);
            ax = ay = az = make_float2(0.f, 0.f);
        }
    }
    if (tt < nt) {
        // the 1PN term is -c^-2 P, the 2PN + 2.5PN term -c^-4 Q (pn.cuh)
        const double c2 = -(double)pk.c2, c4 = -(double)pk.c4;
        store_result(tt, bi, cx.value() + (c2 * (double)(px.x + px.y) + c4 * (double)(qx.x + qx.y)),
                     cy.value() + (c2 * (double)(py.x + py.y) + c4 * (double)(qy.x + qy.y)),
                     cz.value() + (c2 * (double)(pz.x + pz.y) + c4 * (double)(qz.x + qz.y)), Gd, nslices, slice, nt,
                     partial, acc, out3, kick);
    }
}

// Newtonian mixed path with the paired FP32 instructions of sm_100
// (add/mul/fma .f32x2): two j bodies per instruction. The j-tile is staged
// pair-interleaved so every paired operand is an aligned register pair:
//   pa = (hx0, hx1, hy0, hy1)  pb = (hz0, hz1, m0, m1)
//   pc = (lx0, lx1, ly0, ly1)  pd = (lz0, lz1, -, -)
// Same arithmetic per pair as k_allpairs_mixed (double-single separation, SFU
// rsqrt, FP32 partials folded into compensated sums every FOLD j).
template <bool GUARD>
__global__ void __launch_bounds__(BLOCK) k_allpairs_mixed2(
    int64_t j_lo, int64_t n, int64_t nt, const int32_t* __restrict__ targets, const float4* __restrict__ phi,
    const float4* __restrict__ plo, float eps2, double Gd, int64_t slice_len, int nslices,
    double4* __restrict__ partial, double4* __restrict__ acc, double* __restrict__ out3, KickArgs kick) {
    __shared__ float4 pa[BLOCK / 2], pb[BLOCK / 2], pc[BLOCK / 2], pd[BLOCK / 2];
    const int slice = blockIdx.y;
    const int64_t j0 = j_lo + (int64_t)slice * slice_len;  // sources [j_lo, n), sliced
    const int64_t j1 = min(n, j0 + slice_len);
    int64_t tt[IPT], bi[IPT];
    float2 nhx[IPT], nhy[IPT], nhz[IPT], nlx[IPT], nly[IPT], nlz[IPT];
    float2 ax[IPT], ay[IPT], az[IPT];
    CompSum cx[IPT], cy[IPT], cz[IPT];
    const float2 e2 = make_float2(eps2, eps2);
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        tt[k] = (int64_t)blockIdx.x * BLOCK * IPT + k * BLOCK + threadIdx.x;
        bi[k] = tt[k] < nt ? (targets ? (int64_t)targets[tt[k]] : tt[k]) : 0;
        const float4 h = phi[bi[k]], l = plo[bi[k]];
        nhx[k] = make_float2(-h.x, -h.x); nhy[k] = make_float2(-h.y, -h.y); nhz[k] = make_float2(-h.z, -h.z);
        nlx[k] = make_float2(-l.x, -l.x); nly[k] = make_float2(-l.y, -l.y); nlz[k] = make_float2(-l.z, -l.z);
        ax[k] = ay[k] = az[k] = make_float2(0.f, 0.f);
    }
    float* fa = reinterpret_cast<float*>(pa);
    float* fb = reinterpret_cast<float*>(pb);
    float* fc = reinterpret_cast<float*>(pc);
    float* fd = reinterpret_cast<float*>(pd);
    const int q = threadIdx.x >> 1, hh = threadIdx.x & 1;
    for (int64_t base = j0; base < j1; base += BLOCK) {
        const int64_t j = base + threadIdx.x;
        __syncthreads();
        float4 h = make_float4(PAD_POS, PAD_POS, PAD_POS, 0.f), l = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j < j1) { h = phi[j]; l = plo[j]; }
        fa[4 * q + hh] = h.x; fa[4 * q + 2 + hh] = h.y;
        fb[4 * q + hh] = h.z; fb[4 * q + 2 + hh] = h.w;
        fc[4 * q + hh] = l.x; fc[4 * q + 2 + hh] = l.y;
        fd[4 * q + hh] = l.z; fd[4 * q + 2 + hh] = 0.f;
        __syncthreads();
        auto pair2 = [&](int pq) {
            const float4 A = pa[pq], B = pb[pq], C = pc[pq], D = pd[pq];
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                const float2 dx = __fadd2_rn(__fadd2_rn(make_float2(A.x, A.y), nhx[k]), __fadd2_rn(make_float2(C.x, C.y), nlx[k]));
                const float2 dy = __fadd2_rn(__fadd2_rn(make_float2(A.z, A.w), nhy[k]), __fadd2_rn(make_float2(C.z, C.w), nly[k]));
                const float2 dz = __fadd2_rn(__fadd2_rn(make_float2(B.x, B.y), nhz[k]), __fadd2_rn(make_float2(D.x, D.y), nlz[k]));
                float2 r2 = __ffma2_rn(dz, dz, e2);
                r2 = __ffma2_rn(dy, dy, r2);
                r2 = __ffma2_rn(dx, dx, r2);
                float2 inv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                if (GUARD) {
                    inv.x = r2.x > 0.f ? inv.x : 0.f;
                    inv.y = r2.y > 0.f ? inv.y : 0.f;
                }
                const float2 inv2 = __fmul2_rn(inv, inv);
                const float2 s = __fmul2_rn(__fmul2_rn(make_float2(B.z, B.w), inv), inv2);
                ax[k] = __ffma2_rn(dx, s, ax[k]);
                ay[k] = __ffma2_rn(dy, s, ay[k]);
                az[k] = __ffma2_rn(dz, s, az[k]);
            }
        };
        // a partial last tile stops at its last source pair (the padding pairs
        // contribute zero)
        const int npair = (int)((min((int64_t)BLOCK, j1 - base) + 1) / 2);
#pragma unroll 1
        for (int c0 = 0; c0 < npair; c0 += FOLD / 2) {
            if (npair == BLOCK / 2) {
#pragma unroll 8
                for (int pq = c0; pq < c0 + FOLD / 2; ++pq) pair2(pq);
            } else {
#pragma unroll 1
                for (int pq = c0; pq < min(c0 + FOLD / 2, npair); ++pq) pair2(pq);
            }
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                cx[k].add(ax[k].x + ax[k].y); cy[k].add(ay[k].x + ay[k].y); cz[k].add(az[k].x + az[k].y);
                ax[k] = ay[k] = az[k] = make_float2(0.f, 0.f);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k)
        if (tt[k] < nt)
            store_result(tt[k], bi[k], cx[k].value(), cy[k].value(), cz[k].value(), Gd, nslices, slice, nt, partial,
                         acc, out3, kick);
}

__global__ void k_reduce_slices(int64_t nt, int nslices, const double4* __restrict__ partial,
                                const int32_t* __restrict__ targets, double G, double4* __restrict__ acc,
                                double* __restrict__ out3, KickArgs kick) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x) {
        double ax = 0, ay = 0, az = 0;
        for (int s = 0; s < nslices; ++s) {
            double4 p = partial[(int64_t)s * nt + t];
            ax += p.x; ay += p.y; az += p.z;
        }
        int64_t body = targets ? (int64_t)targets[t] : t;
        store_result(t, body, ax, ay, az, G, 1, 0, nt, nullptr, acc, out3, kick);
    }
}

template <int PNL, bool GUARD>
void launch_fp64(dim3 grid, cudaStream_t st, int64_t j_lo, int64_t n, int64_t nt, const int32_t* tg, aster_ctx* c,
                 const aster_params* p, int64_t slice_len, int ns, double4* partial, double* out3, KickArgs kick) {
    k_allpairs_fp64<PNL, GUARD><<<grid, BLOCK, 0, st>>>(j_lo, n, nt, tg, c->pm.as<double4>(), c->vel.as<double4>(), p->G,
                                                         p->eps2, make_pn(p), slice_len, ns, partial,
                                                         c->acc.as<double4>(), out3, kick);
}

template <int PNL, bool GUARD>
void launch_mixed(dim3 grid, cudaStream_t st, int64_t j_lo, int64_t n, int64_t nt, const int32_t* tg, aster_ctx* c,
                  const aster_params* p, int64_t slice_len, int ns, double4* partial, double* out3, KickArgs kick) {
    if constexpr (PNL == 0) {
        k_allpairs_mixed2<GUARD><<<grid, BLOCK, 0, st>>>(j_lo, n, nt, tg, c->phi.as<float4>(), c->plo.as<float4>(),
                                                          (float)p->eps2, p->G, slice_len, ns, partial,
                                                          c->acc.as<double4>(), out3, kick);
    } else {
        k_allpairs_mixed_pn<PNL, GUARD><<<grid, BLOCK, 0, st>>>(
            j_lo, n, nt, tg, c->phi.as<float4>(), c->plo.as<float4>(), c->vf.as<float4>(), (float)p->G, (float)p->eps2,
            pn_float(make_pn(p)), p->G, slice_len, ns, partial, c->acc.as<double4>(), out3, kick);
    }
}

template <int PNL>
void launch_pnl(int precision, bool guard, dim3 grid, cudaStream_t st, int64_t j_lo, int64_t n, int64_t nt,
                const int32_t* tg,
                aster_ctx* c, const aster_params* p, int64_t slice_len, int ns, double4* partial, double* out3,
                KickArgs kick) {
    if (precision == ASTER_FP64) {
        if (guard) launch_fp64<PNL, true>(grid, st, j_lo, n, nt, tg, c, p, slice_len, ns, partial, out3, kick);
        else       launch_fp64<PNL, false>(grid, st, j_lo, n, nt, tg, c, p, slice_len, ns, partial, out3, kick);
    } else {
        if (guard) launch_mixed<PNL, true>(grid, st, j_lo, n, nt, tg, c, p, slice_len, ns, partial, out3, kick);
        else       launch_mixed<PNL, false>(grid, st, j_lo, n, nt, tg, c, p, slice_len, ns, partial, out3, kick);
    }
}

}  // namespace

// Launch one all-pairs evaluation. Targets: every body (targets_dev == null,
// nt == n) or an explicit list. Output: ctx->acc (out_dev == null) with an
// optional closing kick, or out_dev[nt*3].
// Launch one all-pairs evaluation over the sources [src_lo, src_hi) (bodies
// beyond the last massive one are dropped: they attract nothing under any of
// the force laws). Targets: every body (targets_dev == null, nt == n) or an
// explicit list. Output: ctx->acc (out_dev == null) with an optional closing
// kick, or out_dev[nt*3].
int aster_allpairs_launch_range(aster_ctx* c, const aster_params* p, int precision, bool closing_kick, int64_t nt,
                                const int32_t* targets_dev, double* out_dev, int64_t src_lo, int64_t src_hi) {
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    if (precision == ASTER_MIXED && !c->mixed_valid) ASTER_TRY(aster_refresh_mixed(c));
    const int64_t n_src = c->n_src > 0 ? c->n_src : c->n;
    const int64_t lo = src_lo, hi = src_hi < n_src ? src_hi : n_src;
    const int64_t len = hi > lo ? hi - lo : 0;
    // one target per thread in the mixed post-Newtonian kernel, two elsewhere
    const int64_t per_block = (int64_t)BLOCK * (precision == ASTER_MIXED && pn_level(p) > 0 ? IPT_PN : IPT);
    const int64_t iblocks = (nt + per_block - 1) / per_block;
    // j-slices so that small n still fill the GPU (>= ASTER_SLICE_BLOCKS_PER_SM blocks per SM).
    int64_t want = ASTER_SLICE_BLOCKS_PER_SM * (int64_t)c->sm_count;
    int64_t ns = iblocks >= want ? 1 : (want + iblocks - 1) / iblocks;
    // each slice at least one j-tile; the mixed kernel's at least
    // ASTER_SLICE_MIN_MIXED sources (its partial-sum reduction outweighs more
    // parallelism below that)
    const int64_t min_len = precision == ASTER_MIXED ? ASTER_SLICE_MIN_MIXED : BLOCK;
    int64_t max_ns = (len + min_len - 1) / min_len;
    if (ns > max_ns) ns = max_ns;
    if (ns > 64) ns = 64;
    if (ns < 1) ns = 1;
    int64_t slice_len = ((len + ns - 1) / ns + BLOCK - 1) / BLOCK * BLOCK;
    if (slice_len < BLOCK) slice_len = BLOCK;
    ns = (len + slice_len - 1) / slice_len;
    if (ns < 1) ns = 1;  // no sources: one slice that writes zeros
    double4* partial = nullptr;
    if (ns > 1) {
        ASTER_TRY(c->scratch.ensure((size_t)ns * nt * sizeof(double4)));
        partial = c->scratch.as<double4>();
    }
    KickArgs kick{closing_kick && !out_dev, 0.5 * p->dt, c->vel.as<double4>()};
    if (kick.on) c->mixed_valid = false;  // the closing kick moves the velocities
    dim3 grid((unsigned)iblocks, (unsigned)ns);
    const bool guard = !(p->eps2 > 0.0);
    const int pnl = pn_level(p);
    const int64_t j_hi = lo + len;
    if (pnl == 2) launch_pnl<2>(precision, guard, grid, c->stream, lo, j_hi, nt, targets_dev, c, p, slice_len, (int)ns, partial, out_dev, kick);
    else if (pnl == 1) launch_pnl<1>(precision, guard, grid, c->stream, lo, j_hi, nt, targets_dev, c, p, slice_len, (int)ns, partial, out_dev, kick);
    else launch_pnl<0>(precision, guard, grid, c->stream, lo, j_hi, nt, targets_dev, c, p, slice_len, (int)ns, partial, out_dev, kick);
    ASTER_CUDA(cudaGetLastError());
    c->stats.kernels += 1;
    if (ns > 1) {
        int g = (int)((nt + 255) / 256);
        k_reduce_slices<<<g, 256, 0, c->stream>>>(nt, (int)ns, partial, targets_dev, p->G, c->acc.as<double4>(),
                                                  out_dev, kick);
        ASTER_CUDA(cudaGetLastError());
        c->stats.kernels += 1;
    }
    c->stats.interactions += (double)nt * (double)len;
    return ASTER_OK;
}

// Every source body [0, n).
int aster_allpairs_launch(aster_ctx* c, const aster_params* p, int precision, bool closing_kick, int64_t nt,
                          const int32_t* targets_dev, double* out_dev) {
    return aster_allpairs_launch_range(c, p, precision, closing_kick, nt, targets_dev, out_dev, 0, c->n);
}

extern "C" int aster_allpairs(aster_ctx* c, const aster_params* p, int precision, double* acc_out) {
    if (!c) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    cudaEventRecord(c->ev[0], c->stream);
    ASTER_TRY(aster_allpairs_launch(c, p, precision, false, c->n, nullptr, nullptr));
    cudaEventRecord(c->ev[1], c->stream);
    ASTER_TRY(aster_finish(c));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = c->stats.ms_force = ms;
    c->acc_valid = true;
    return aster_copy_acc_out(c, acc_out);
}

// Accelerations of every body from the sources [src_lo, src_hi) only
// (src_hi < 0: up to n), as Parallelized::compute_forces sums over the
// solver's set_bounds range. The cached acceleration is not the full one
// afterwards, so the next KDK step evaluates it afresh.
extern "C" int aster_allpairs_range(aster_ctx* c, const aster_params* p, int precision, int64_t src_lo,
                                    int64_t src_hi, double* acc_out) {
    if (!c) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    if (src_hi < 0) src_hi = c->n;
    if (src_lo < 0 || src_lo > src_hi || src_hi > c->n) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    cudaEventRecord(c->ev[0], c->stream);
    ASTER_TRY(aster_allpairs_launch_range(c, p, precision, false, c->n, nullptr, nullptr, src_lo, src_hi));
    cudaEventRecord(c->ev[1], c->stream);
    ASTER_TRY(aster_finish(c));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = c->stats.ms_force = ms;
    c->acc_valid = false;
    return aster_copy_acc_out(c, acc_out);
}

extern "C" int aster_allpairs_targets(aster_ctx* c, const aster_params* p, int precision, int64_t nt,
                                      const int32_t* targets, double* acc_out) {
    if (!c || !targets || !acc_out || nt <= 0) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    for (int64_t t = 0; t < nt; ++t)
        if (targets[t] < 0 || targets[t] >= c->n) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_begin(c));
    ASTER_TRY(c->targets.ensure((size_t)nt * sizeof(int32_t) + (size_t)nt * 3 * sizeof(double) + 256));
    int32_t* tg = c->targets.as<int32_t>();
    double* out = reinterpret_cast<double*>(c->targets.as<char>() + ((nt * sizeof(int32_t) + 255) / 256) * 256);
    ASTER_CUDA(cudaMemcpyAsync(tg, targets, (size_t)nt * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    ASTER_TRY(aster_allpairs_launch(c, p, precision, false, nt, tg, out));
    ASTER_CUDA(cudaMemcpyAsync(acc_out, out, (size_t)nt * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return aster_finish(c);
}
