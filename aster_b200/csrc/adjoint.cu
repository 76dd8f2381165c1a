// Adjoint (reverse mode) of the kick-drift-kick leapfrog with checkpointed
// recomputation. The reference has no differentiation; the forward map is the
// one aster_kdk_steps integrates (update_leapfrog's map,
// src/physics/tool_chain_impl.cpp:169-185, one force evaluation per step).
//
// Forward step n (h = dt/2, A(x) the softened Newtonian acceleration):
//   v' = v_n + h A(x_n);  x_{n+1} = x_n + dt v';  v_{n+1} = v' + h A(x_{n+1})
// Reverse sweep for L = (1/N) sum |x_T - x*|^2 (lx = dL/dx, lv = dL/dv):
//   seed lx = (2/N)(x_T - x*), lv = 0, lm = 0; for n = T-1 .. 0:
//     lv' = lv + dt lx;  w = c_n h lv';  lx += J(x_n)^T w;  lm += (dA/dm)^T w;  lv = lv'
//   with c_n = 2 (A(x_n) feeds the closing kick of step n-1 and the opening
//   kick of step n with the same cotangent) except c_0 = 1.
// The O(N^2) part, per pair (k target, j source, d = x_j - x_k,
// s = (d.d + eps2)^(-1/2), u = m_k w_j - m_j w_k):
//   (J^T w)_k += G [ s^3 u - 3 s^5 d (d.u) ];  (dA/dm)^T w at k += -G s^3 (w_j . d)
// tiled like the all-pairs force (double-single separations and compensated
// sums in the mixed path).
//
// Memory: (x, v, a) every K steps (checkpoints) and the K+1 positions of the
// segment being reversed; the segment is recomputed from its checkpoint with
// the same kernels, so it reproduces the forward pass bit for bit.
#include <algorithm>
#include <cmath>

#include "aster_internal.cuh"

namespace {

constexpr int BLOCK = 128;
constexpr int IPT = 2;
constexpr int FOLD = 64;

__global__ void k_adj_seed(int64_t n, const double4* __restrict__ pm, const double* __restrict__ target,
                           double4* __restrict__ lx, double4* __restrict__ lv, double* __restrict__ lm,
                           double* __restrict__ part) {
    __shared__ double red[8];
    double s = 0.0;
    const double inv_n = 1.0 / (double)n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 x = pm[i];
        const double dx = x.x - target[3 * i], dy = x.y - target[3 * i + 1], dz = x.z - target[3 * i + 2];
        s += dx * dx + dy * dy + dz * dz;
        lx[i] = make_double4(2.0 * inv_n * dx, 2.0 * inv_n * dy, 2.0 * inv_n * dz, 0.0);
        lv[i] = make_double4(0, 0, 0, 0);
        lm[i] = 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

__global__ void k_adj_loss_final(int nb, const double* __restrict__ part, double inv_n, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t = 0;
        for (int b = 0; b < nb; ++b) t += part[b];
        out[0] = t * inv_n;
    }
}

// lv' = lv + dt lx; w = scale * lv'; lv = lv'
template <bool MIXED>
__global__ void k_adj_pre(int64_t n, const double4* __restrict__ lx, double4* __restrict__ lv, void* __restrict__ w_out,
                          double dt, double scale) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 a = lx[i];
        double4 v = lv[i];
        v.x += dt * a.x; v.y += dt * a.y; v.z += dt * a.z;
        lv[i] = v;
        if (MIXED)
            static_cast<float4*>(w_out)[i] = make_float4((float)(scale * v.x), (float)(scale * v.y),
                                                          (float)(scale * v.z), 0.f);
        else
            static_cast<double4*>(w_out)[i] = make_double4(scale * v.x, scale * v.y, scale * v.z, 0.0);
    }
}

// Result for target k: add G * (jt, g) to lx[k], lm[k] or write slice partials.
__device__ __forceinline__ void adj_store(int64_t k, double jx, double jy, double jz, double g, double G,
                                          int nslices, int slice, int64_t n, double4* __restrict__ partial,
                                          double4* __restrict__ lx, double* __restrict__ lm) {
    if (nslices > 1) {
        partial[(int64_t)slice * n + k] = make_double4(jx, jy, jz, g);
        return;
    }
    double4 a = lx[k];
    a.x += G * jx; a.y += G * jy; a.z += G * jz;
    lx[k] = a;
    lm[k] += G * g;
}

// Mixed adjoint pair terms, two sources at once with the paired FP32
// instructions of sm_100 (add/mul/fma .f32x2): the source tile is stored
// pair-interleaved, element k of each array holding sources 2k and 2k + 1, so
// every paired operand is one aligned register pair. Per target (IPT per
// thread) the FP32 partial sums are folded into compensated accumulators
// every FOLD sources; the mass-gradient sum is kept positive (s^3 w_j.d) and
// negated at the fold.
template <bool GUARD>
__global__ void __launch_bounds__(BLOCK) k_adj_pair_mixed(int64_t n, const double4* __restrict__ xs,
                                                          const float4* __restrict__ w, float eps2, double G,
                                                          int64_t slice_len, int nslices,
                                                          double4* __restrict__ partial, double4* __restrict__ lx,
                                                          double* __restrict__ lm) {
    constexpr int NP = BLOCK / 2;
    __shared__ float4 PA[NP], PB[NP], PC[NP], PD[NP], PE[NP];  // (x_hi x_hi' y_hi y_hi'), (z_hi z_hi' m m'),
                                                               // (x_lo ..), (z_lo z_lo' w_z w_z'), (w_x .. w_y ..)
    const int slice = blockIdx.y;
    const int64_t j0 = (int64_t)slice * slice_len, j1 = min(n, j0 + slice_len);
    int64_t kk[IPT];
    float2 nxh[IPT], nyh[IPT], nzh[IPT], nxl[IPT], nyl[IPT], nzl[IPT], mk[IPT], nwx[IPT], nwy[IPT], nwz[IPT];
    float2 ax[IPT], ay[IPT], az[IPT], ag[IPT];
    CompSum cx[IPT], cy[IPT], cz[IPT], cg[IPT];
    const float2 zero2 = make_float2(0.f, 0.f), e2 = make_float2(eps2, eps2);
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
        kk[q] = (int64_t)blockIdx.x * BLOCK * IPT + q * BLOCK + threadIdx.x;
        const int64_t k = kk[q] < n ? kk[q] : 0;
        const double4 x = xs[k];
        float h, l;
        ds_split(x.x, h, l); nxh[q] = make_float2(-h, -h); nxl[q] = make_float2(-l, -l);
        ds_split(x.y, h, l); nyh[q] = make_float2(-h, -h); nyl[q] = make_float2(-l, -l);
        ds_split(x.z, h, l); nzh[q] = make_float2(-h, -h); nzl[q] = make_float2(-l, -l);
        const float m = (float)x.w;
        mk[q] = make_float2(m, m);
        const float4 wk = w[k];
        nwx[q] = make_float2(-wk.x, -wk.x); nwy[q] = make_float2(-wk.y, -wk.y); nwz[q] = make_float2(-wk.z, -wk.z);
        ax[q] = ay[q] = az[q] = ag[q] = zero2;
    }
    for (int64_t base = j0; base < j1; base += BLOCK) {
        const int64_t j = base + threadIdx.x;
        __syncthreads();
        {
            float hx, lx_, hy, ly, hz, lz, m = 0.f;
            float4 wj = make_float4(0.f, 0.f, 0.f, 0.f);
            if (j < j1) {
                const double4 x = xs[j];
                ds_split(x.x, hx, lx_);
                ds_split(x.y, hy, ly);
                ds_split(x.z, hz, lz);
                m = (float)x.w;
                wj = w[j];
            } else {  // far away, no mass, no cotangent: contributes nothing
                hx = hy = hz = 1.0e30f;
                lx_ = ly = lz = 0.f;
            }
            const int o = ((threadIdx.x >> 1) << 2) | (threadIdx.x & 1);
            float* A = reinterpret_cast<float*>(PA);
            float* B = reinterpret_cast<float*>(PB);
            float* C = reinterpret_cast<float*>(PC);
            float* D = reinterpret_cast<float*>(PD);
            float* E = reinterpret_cast<float*>(PE);
            A[o] = hx; A[o + 2] = hy; B[o] = hz; B[o + 2] = m;
            C[o] = lx_; C[o + 2] = ly; D[o] = lz; D[o + 2] = wj.z;
            E[o] = wj.x; E[o + 2] = wj.y;
        }
        __syncthreads();
#pragma unroll 1
        for (int c0 = 0; c0 < NP; c0 += FOLD / 2) {
#pragma unroll 4
            for (int pp = c0; pp < c0 + FOLD / 2; ++pp) {
                const float4 a = PA[pp], b = PB[pp], c = PC[pp], d = PD[pp], e = PE[pp];
                const float2 mj = make_float2(b.z, b.w);
                const float2 wjx = make_float2(e.x, e.y), wjy = make_float2(e.z, e.w), wjz = make_float2(d.z, d.w);
#pragma unroll
                for (int q = 0; q < IPT; ++q) {
                    const float2 dx = __fadd2_rn(__fadd2_rn(make_float2(a.x, a.y), nxh[q]),
                                                 __fadd2_rn(make_float2(c.x, c.y), nxl[q]));
                    const float2 dy = __fadd2_rn(__fadd2_rn(make_float2(a.z, a.w), nyh[q]),
                                                 __fadd2_rn(make_float2(c.z, c.w), nyl[q]));
                    const float2 dz = __fadd2_rn(__fadd2_rn(make_float2(b.x, b.y), nzh[q]),
                                                 __fadd2_rn(make_float2(d.x, d.y), nzl[q]));
                    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
                    float2 sv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                    if (GUARD) {
                        sv.x = r2.x > 0.f ? sv.x : 0.f;
                        sv.y = r2.y > 0.f ? sv.y : 0.f;
                    }
                    const float2 s2 = __fmul2_rn(sv, sv), s3 = __fmul2_rn(s2, sv);
                    // u = m_k w_j - m_j w_k
                    const float2 ux = __ffma2_rn(mk[q], wjx, __fmul2_rn(mj, nwx[q]));
                    const float2 uy = __ffma2_rn(mk[q], wjy, __fmul2_rn(mj, nwy[q]));
                    const float2 uz = __ffma2_rn(mk[q], wjz, __fmul2_rn(mj, nwz[q]));
                    const float2 du = __ffma2_rn(dx, ux, __ffma2_rn(dy, uy, __fmul2_rn(dz, uz)));
                    // s^3 u - 3 s^5 (d.u) d = s^3 (u + k d), k = -3 s^2 (d.u)
                    const float2 k = __fmul2_rn(__fmul2_rn(s2, du), make_float2(-3.f, -3.f));
                    ax[q] = __ffma2_rn(s3, __ffma2_rn(k, dx, ux), ax[q]);
                    ay[q] = __ffma2_rn(s3, __ffma2_rn(k, dy, uy), ay[q]);
                    az[q] = __ffma2_rn(s3, __ffma2_rn(k, dz, uz), az[q]);
                    const float2 wd = __ffma2_rn(wjx, dx, __ffma2_rn(wjy, dy, __fmul2_rn(wjz, dz)));
                    ag[q] = __ffma2_rn(s3, wd, ag[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < IPT; ++q) {
                cx[q].add(ax[q].x + ax[q].y); cy[q].add(ay[q].x + ay[q].y); cz[q].add(az[q].x + az[q].y);
                cg[q].add(-(ag[q].x + ag[q].y));
                ax[q] = ay[q] = az[q] = ag[q] = zero2;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < IPT; ++q)
        if (kk[q] < n)
            adj_store(kk[q], cx[q].value(), cy[q].value(), cz[q].value(), cg[q].value(), G, nslices, slice, n, partial,
                      lx, lm);
}

template <bool GUARD>
__global__ void __launch_bounds__(BLOCK) k_adj_pair_fp64(int64_t n, const double4* __restrict__ xs,
                                                         const double4* __restrict__ w, double eps2, double G,
                                                         int64_t slice_len, int nslices,
                                                         double4* __restrict__ partial, double4* __restrict__ lx,
                                                         double* __restrict__ lm) {
    __shared__ double4 sx[BLOCK], sw[BLOCK];
    const int slice = blockIdx.y;
    const int64_t j0 = (int64_t)slice * slice_len, j1 = min(n, j0 + slice_len);
    int64_t kk[IPT];
    double4 xk[IPT], wk[IPT];
    double ax[IPT], ay[IPT], az[IPT], ag[IPT];
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
        kk[q] = (int64_t)blockIdx.x * BLOCK * IPT + q * BLOCK + threadIdx.x;
        const int64_t k = kk[q] < n ? kk[q] : 0;
        xk[q] = xs[k];
        wk[q] = w[k];
        ax[q] = ay[q] = az[q] = ag[q] = 0.0;
    }
    for (int64_t base = j0; base < j1; base += BLOCK) {
        const int64_t j = base + threadIdx.x;
        __syncthreads();
        sx[threadIdx.x] = j < j1 ? xs[j] : make_double4(1e300, 1e300, 1e300, 0.0);
        sw[threadIdx.x] = j < j1 ? w[j] : make_double4(0, 0, 0, 0);
        __syncthreads();
#pragma unroll 4
        for (int jj = 0; jj < BLOCK; ++jj) {
            const double4 xj = sx[jj], wj = sw[jj];
#pragma unroll
            for (int q = 0; q < IPT; ++q) {
                const double dx = xj.x - xk[q].x, dy = xj.y - xk[q].y, dz = xj.z - xk[q].z;
                const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
                double s = rsqrt(r2);
                if (GUARD) s = r2 > 0.0 ? s : 0.0;
                const double s2 = s * s, s3 = s2 * s, s5 = s3 * s2;
                const double ux = xk[q].w * wj.x - xj.w * wk[q].x;
                const double uy = xk[q].w * wj.y - xj.w * wk[q].y;
                const double uz = xk[q].w * wj.z - xj.w * wk[q].z;
                const double du = dx * ux + dy * uy + dz * uz;
                const double t = 3.0 * s5 * du;
                ax[q] += s3 * ux - t * dx;
                ay[q] += s3 * uy - t * dy;
                az[q] += s3 * uz - t * dz;
                ag[q] -= s3 * (wj.x * dx + wj.y * dy + wj.z * dz);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < IPT; ++q)
        if (kk[q] < n) adj_store(kk[q], ax[q], ay[q], az[q], ag[q], G, nslices, slice, n, partial, lx, lm);
}

__global__ void k_adj_reduce(int64_t n, int nslices, const double4* __restrict__ partial, double G,
                             double4* __restrict__ lx, double* __restrict__ lm) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double jx = 0, jy = 0, jz = 0, g = 0;
        for (int s = 0; s < nslices; ++s) {
            const double4 p = partial[(int64_t)s * n + k];
            jx += p.x; jy += p.y; jz += p.z; g += p.w;
        }
        adj_store(k, jx, jy, jz, g, G, 1, 0, n, nullptr, lx, lm);
    }
}

__global__ void k_unpack_d4(int64_t n, const double4* __restrict__ src, double* __restrict__ dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 v = src[i];
        dst[3 * i] = v.x; dst[3 * i + 1] = v.y; dst[3 * i + 2] = v.z;
    }
}

int adj_pair_launch(aster_ctx* c, const aster_params* p, int precision, const double4* xs) {
    AdjBufs& a = c->adj;
    const int64_t n = c->n;
    const int64_t iblocks = (n + BLOCK * IPT - 1) / (BLOCK * IPT);
    int64_t want = ASTER_SLICE_BLOCKS_PER_SM * (int64_t)c->sm_count;
    int64_t ns = iblocks >= want ? 1 : (want + iblocks - 1) / iblocks;
    const int64_t max_ns = (n + BLOCK - 1) / BLOCK;
    ns = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(ns, max_ns), 64));
    const int64_t slice_len = ((n + ns - 1) / ns + BLOCK - 1) / BLOCK * BLOCK;
    ns = (n + slice_len - 1) / slice_len;
    double4* partial = nullptr;
    if (ns > 1) {
        ASTER_TRY(a.part.ensure((size_t)ns * n * sizeof(double4)));
        partial = a.part.as<double4>();
    }
    const dim3 grid((unsigned)iblocks, (unsigned)ns);
    const bool guard = !(p->eps2 > 0.0);
    if (precision == ASTER_MIXED) {
        if (guard)
            k_adj_pair_mixed<true><<<grid, BLOCK, 0, c->stream>>>(n, xs, a.w.as<float4>(), (float)p->eps2, p->G,
                                                                 slice_len, (int)ns, partial, a.lx.as<double4>(),
                                                                 a.lm.as<double>());
        else
            k_adj_pair_mixed<false><<<grid, BLOCK, 0, c->stream>>>(n, xs, a.w.as<float4>(), (float)p->eps2, p->G,
                                                                  slice_len, (int)ns, partial, a.lx.as<double4>(),
                                                                  a.lm.as<double>());
    } else {
        if (guard)
            k_adj_pair_fp64<true><<<grid, BLOCK, 0, c->stream>>>(n, xs, a.w.as<double4>(), p->eps2, p->G, slice_len,
                                                                (int)ns, partial, a.lx.as<double4>(),
                                                                a.lm.as<double>());
        else
            k_adj_pair_fp64<false><<<grid, BLOCK, 0, c->stream>>>(n, xs, a.w.as<double4>(), p->eps2, p->G,
                                                                 slice_len, (int)ns, partial, a.lx.as<double4>(),
                                                                 a.lm.as<double>());
    }
    ASTER_CUDA(cudaGetLastError());
    c->stats.kernels += 1;
    if (ns > 1) {
        k_adj_reduce<<<(int)((n + 255) / 256), 256, 0, c->stream>>>(n, (int)ns, partial, p->G, a.lx.as<double4>(),
                                                                  a.lm.as<double>());
        ASTER_CUDA(cudaGetLastError());
        c->stats.kernels += 1;
    }
    return ASTER_OK;
}

// One forward KDK step of the context state (the aster_kdk_steps step).
int forward_step(aster_ctx* c, const aster_params* p, int precision) {
    ASTER_TRY(aster_kick_drift_launch(c, p, false, precision == ASTER_MIXED));
    return aster_allpairs_launch(c, p, precision, true, c->n, nullptr, nullptr);
}

int copy_d2d(aster_ctx* c, void* dst, const void* src, size_t bytes) {
    ASTER_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
    return ASTER_OK;
}

}  // namespace

extern "C" int aster_adjoint_leapfrog(aster_ctx* c, const aster_params* p, int precision, int64_t nsteps,
                                      int32_t K, const double* target, double* loss, double* grad_x0,
                                      double* grad_v0, double* grad_m) {
    if (!c || !target || nsteps < 1 || K < 1) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    if (p->force_law & (ASTER_PN1 | ASTER_PN2 | ASTER_PN25)) return ASTER_ERR_UNSUPPORTED;
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    AdjBufs& a = c->adj;
    const int64_t n = c->n;
    const size_t v4 = (size_t)n * sizeof(double4);
    const int64_t nseg = (nsteps + K - 1) / K;
    ASTER_TRY(a.ckpt.ensure((size_t)nseg * 3 * v4));
    ASTER_TRY(a.segx.ensure((size_t)(K + 1) * v4));
    ASTER_TRY(a.lx.ensure(v4));
    ASTER_TRY(a.lv.ensure(v4));
    ASTER_TRY(a.lm.ensure((size_t)n * sizeof(double)));
    ASTER_TRY(a.w.ensure(v4));
    ASTER_TRY(a.target.ensure((size_t)n * 3 * sizeof(double)));
    ASTER_TRY(c->red.ensure(4096));
    const int nb = (int)std::min<int64_t>((n + 255) / 256, 1024);
    ASTER_TRY(c->scratch.ensure((size_t)nb * sizeof(double) + 64));
    ASTER_CUDA(cudaMemcpyAsync(a.target.ptr, target, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice,
                               c->stream));
    char* ck = a.ckpt.as<char>();
    auto ck_x = [&](int64_t s) { return ck + (size_t)s * 3 * v4; };
    auto ck_v = [&](int64_t s) { return ck + (size_t)s * 3 * v4 + v4; };
    auto ck_a = [&](int64_t s) { return ck + (size_t)s * 3 * v4 + 2 * v4; };
    const double h = 0.5 * p->dt;
    cudaEventRecord(c->ev[0], c->stream);

    // forward pass with checkpoints
    if (precision == ASTER_MIXED) ASTER_TRY(aster_refresh_mixed(c));
    ASTER_TRY(aster_allpairs_launch(c, p, precision, false, n, nullptr, nullptr));  // a(x0)
    for (int64_t s = 0; s < nsteps; ++s) {
        if (s % K == 0) {
            ASTER_TRY(copy_d2d(c, ck_x(s / K), c->pm.ptr, v4));
            ASTER_TRY(copy_d2d(c, ck_v(s / K), c->vel.ptr, v4));
            ASTER_TRY(copy_d2d(c, ck_a(s / K), c->acc.ptr, v4));
        }
        ASTER_TRY(forward_step(c, p, precision));
    }
    // loss and seeds
    k_adj_seed<<<nb, 256, 0, c->stream>>>(n, c->pm.as<double4>(), a.target.as<double>(), a.lx.as<double4>(),
                                          a.lv.as<double4>(), a.lm.as<double>(), c->scratch.as<double>());
    ASTER_CUDA(cudaGetLastError());
    double* loss_dev = red_energy(c) + 4;
    k_adj_loss_final<<<1, 32, 0, c->stream>>>(nb, c->scratch.as<double>(), 1.0 / (double)n, loss_dev);
    ASTER_CUDA(cudaGetLastError());

    // reverse pass, segment by segment
    const int eg = (int)std::min<int64_t>((n + 255) / 256, (int64_t)c->sm_count * 8);
    for (int64_t seg = nseg - 1; seg >= 0; --seg) {
        const int64_t start = seg * K, len = std::min<int64_t>(K, nsteps - start);
        ASTER_TRY(copy_d2d(c, c->pm.ptr, ck_x(seg), v4));
        ASTER_TRY(copy_d2d(c, c->vel.ptr, ck_v(seg), v4));
        ASTER_TRY(copy_d2d(c, c->acc.ptr, ck_a(seg), v4));
        if (precision == ASTER_MIXED) ASTER_TRY(aster_refresh_mixed(c));
        ASTER_TRY(copy_d2d(c, a.segx.ptr, c->pm.ptr, v4));
        for (int64_t t = 0; t + 1 < len; ++t) {  // positions x_start .. x_{start+len-1}
            ASTER_TRY(forward_step(c, p, precision));
            ASTER_TRY(copy_d2d(c, a.segx.as<char>() + (size_t)(t + 1) * v4, c->pm.ptr, v4));
        }
        for (int64_t t = len - 1; t >= 0; --t) {
            const int64_t step = start + t;
            const double scale = (step >= 1 ? 2.0 : 1.0) * h;
            if (precision == ASTER_MIXED)
                k_adj_pre<true><<<eg, 256, 0, c->stream>>>(n, a.lx.as<double4>(), a.lv.as<double4>(), a.w.ptr, p->dt,
                                                           scale);
            else
                k_adj_pre<false><<<eg, 256, 0, c->stream>>>(n, a.lx.as<double4>(), a.lv.as<double4>(), a.w.ptr,
                                                            p->dt, scale);
            ASTER_CUDA(cudaGetLastError());
            ASTER_TRY(adj_pair_launch(c, p, precision, reinterpret_cast<const double4*>(a.segx.as<char>() +
                                                                                        (size_t)t * v4)));
        }
    }
    cudaEventRecord(c->ev[1], c->stream);
    // outputs, then restore the uploaded state (x0, v0, a(x0))
    double loss_h = 0.0;
    ASTER_CUDA(cudaMemcpyAsync(&loss_h, loss_dev, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ASTER_TRY(c->stage.ensure((size_t)n * 6 * sizeof(double)));
    double* st = c->stage.as<double>();
    if (grad_x0) {
        k_unpack_d4<<<eg, 256, 0, c->stream>>>(n, a.lx.as<double4>(), st);
        ASTER_CUDA(cudaMemcpyAsync(grad_x0, st, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    if (grad_v0) {
        k_unpack_d4<<<eg, 256, 0, c->stream>>>(n, a.lv.as<double4>(), st + 3 * n);
        ASTER_CUDA(cudaMemcpyAsync(grad_v0, st + 3 * n, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                   c->stream));
    }
    if (grad_m)
        ASTER_CUDA(cudaMemcpyAsync(grad_m, a.lm.ptr, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ASTER_TRY(copy_d2d(c, c->pm.ptr, ck_x(0), v4));
    ASTER_TRY(copy_d2d(c, c->vel.ptr, ck_v(0), v4));
    ASTER_TRY(copy_d2d(c, c->acc.ptr, ck_a(0), v4));
    ASTER_TRY(aster_refresh_mixed(c));  // double-single copies of the restored state
    const int stt = aster_finish(c);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->acc_valid = stt == ASTER_OK;
    if (loss) *loss = loss_h;
    return stt;
}
