// Device-resident stepping with time series recorded on the device: the
// reference's Simulation::step/integrate with its Graph collectors
// (src/utils/builder_endpoint.cpp:274-352, src/utils/graph_collection.cpp,
// src/utils/collectors.cpp), which read the bodies back to the host every
// step (read_bodies_gpu, builder_endpoint.cpp:424-434) and evaluate each
// collector there. Here the chosen updater advances the resident state `rate`
// steps at a time without synchronising, collector kernels write one row per
// sample into a device table, and the table comes back in one copy at the end.
//
// Columns, in this order for the bits set:
//   ENERGY        hamiltonian_collector: total energy (reference formula
//                 -G m_i m_j / (r + eps2) when ref_form, else Plummer-softened)
//   ENERGY_ERROR  error_collector: |E - E0| / |E0|, E0 at the call's start (the
//                 reference keeps E0 in a function-static across simulations)
//   MOMENTUM      total momentum (3)
//   CENTER        centre of mass (3)
//   DISTANCE      distance_collector per body: |x_cm - x_b + 0.1| (n); the
//                 reference adds 0.1 to every component, as here, but its
//                 get_center_of_mass (builder_endpoint.cpp:262-269) returns
//                 (x_cm, x_cm, x_cm) (it scales mp_sum[0]); the true centre
//                 of mass is used here.
#include <algorithm>

#include "aster_internal.cuh"

namespace {

constexpr int REC_BLOCK = 256;

// block partials of (sum m x, sum m) over all bodies
__global__ void __launch_bounds__(REC_BLOCK) k_rec_com_partial(int64_t n, const double4* __restrict__ pm,
                                                               double* __restrict__ part) {
    double s[4] = {0, 0, 0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 p = pm[i];
        s[0] += p.w * p.x; s[1] += p.w * p.y; s[2] += p.w * p.z; s[3] += p.w;
    }
    __shared__ double red[4][REC_BLOCK / 32];
    for (int k = 0; k < 4; ++k) {
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0;
        for (int w = 0; w < REC_BLOCK / 32; ++w) v += red[threadIdx.x][w];
        part[blockIdx.x * 4 + threadIdx.x] = v;
    }
}

// com4 = (x_cm, y_cm, z_cm, M); fixed summation order
__global__ void k_rec_com_final(int64_t nb, const double* __restrict__ part, double* __restrict__ com4) {
    __shared__ double s[4];
    if (threadIdx.x < 4) {
        double v = 0;
        for (int64_t b = 0; b < nb; ++b) v += part[b * 4 + threadIdx.x];
        s[threadIdx.x] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        com4[0] = s[0] / s[3]; com4[1] = s[1] / s[3]; com4[2] = s[2] / s[3]; com4[3] = s[3];
    }
}

// the scalar columns of one row
__global__ void k_rec_row(double* __restrict__ row, double t, int collect, const double* __restrict__ en4,
                          const double* __restrict__ e0, const double* __restrict__ com4) {
    if (threadIdx.x != 0) return;
    int k = 0;
    row[k++] = t;
    if (collect & ASTER_COLLECT_ENERGY) row[k++] = en4[0];
    if (collect & ASTER_COLLECT_ENERGY_ERROR) row[k++] = fabs(en4[0] - e0[0]) / fabs(e0[0]);
    if (collect & ASTER_COLLECT_MOMENTUM) { row[k++] = en4[1]; row[k++] = en4[2]; row[k++] = en4[3]; }
    if (collect & ASTER_COLLECT_CENTER) { row[k++] = com4[0]; row[k++] = com4[1]; row[k++] = com4[2]; }
}

__global__ void __launch_bounds__(REC_BLOCK) k_rec_distance(int64_t n, const double4* __restrict__ pm,
                                                            const double* __restrict__ com4, double* __restrict__ out) {
    const double cx = com4[0], cy = com4[1], cz = com4[2];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 p = pm[i];
        const double dx = cx - p.x + 0.1, dy = cy - p.y + 0.1, dz = cz - p.z + 0.1;
        out[i] = sqrt(dx * dx + dy * dy + dz * dz);
    }
}

__global__ void k_rec_copy(const double* __restrict__ src, double* __restrict__ dst) {
    if (threadIdx.x == 0) dst[0] = src[0];
}

bool needs_energy(int collect) {
    return (collect & (ASTER_COLLECT_ENERGY | ASTER_COLLECT_ENERGY_ERROR | ASTER_COLLECT_MOMENTUM)) != 0;
}
bool needs_com(int collect) { return (collect & (ASTER_COLLECT_CENTER | ASTER_COLLECT_DISTANCE)) != 0; }

}  // namespace

extern "C" int64_t aster_record_columns(const aster_record_config* cfg, int64_t n) {
    if (!cfg || n < 0) return -1;
    int64_t k = 1;
    if (cfg->collect & ASTER_COLLECT_ENERGY) k += 1;
    if (cfg->collect & ASTER_COLLECT_ENERGY_ERROR) k += 1;
    if (cfg->collect & ASTER_COLLECT_MOMENTUM) k += 3;
    if (cfg->collect & ASTER_COLLECT_CENTER) k += 3;
    if (cfg->collect & ASTER_COLLECT_DISTANCE) k += n;
    return k;
}

extern "C" int aster_record(aster_ctx* c, const aster_params* p, const aster_record_config* cfg, int64_t nsteps,
                            double* rows_out) {
    if (!c || !cfg || !rows_out || nsteps < 0) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    const int all = ASTER_COLLECT_ENERGY | ASTER_COLLECT_ENERGY_ERROR | ASTER_COLLECT_MOMENTUM |
                    ASTER_COLLECT_CENTER | ASTER_COLLECT_DISTANCE;
    if (cfg->rate < 1 || (cfg->collect & ~all) || cfg->reserved != 0) return ASTER_ERR_INVALID_ARG;
    if (cfg->updater != ASTER_UPDATER_KDK && cfg->updater != ASTER_UPDATER_SABA && cfg->updater != ASTER_UPDATER_WH)
        return ASTER_ERR_INVALID_ARG;
    if (nsteps > (int64_t)INT32_MAX) return ASTER_ERR_TOO_LARGE;
    const int64_t n = c->n;
    const int64_t ncol = aster_record_columns(cfg, n);
    const int64_t nsamp = nsteps / cfg->rate + 1;
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    const int64_t nbe = aster_energy_parts(c);                                              // energy partials
    const int64_t nbc = std::min<int64_t>((n + REC_BLOCK - 1) / REC_BLOCK, (int64_t)c->sm_count * 4);  // com
    const size_t table = (size_t)(nsamp * ncol);
    ASTER_TRY(c->rec.ensure((table + (size_t)nbe * 5 + (size_t)nbc * 4 + 16) * sizeof(double)));
    double* rows = c->rec.as<double>();
    double* epart = rows + table;
    double* cpart = epart + nbe * 5;
    double* en4 = cpart + nbc * 4;
    double* com4 = en4 + 4;
    double* e0 = com4 + 4;
    double m0 = 0.0;
    if (cfg->updater == ASTER_UPDATER_WH) ASTER_TRY(aster_wh_central_mass(c, &m0));
    const int cgrid = (int)(nbc < 1 ? 1 : nbc);
    auto sample = [&](int64_t k, double t) -> int {
        double* row = rows + k * ncol;
        if (needs_energy(cfg->collect)) ASTER_TRY(aster_energy_enqueue(c, p, cfg->ref_form, epart, en4));
        if (needs_com(cfg->collect)) {
            k_rec_com_partial<<<cgrid, REC_BLOCK, 0, c->stream>>>(n, c->pm.as<double4>(), cpart);
            k_rec_com_final<<<1, 32, 0, c->stream>>>(cgrid, cpart, com4);
        }
        if (k == 0 && needs_energy(cfg->collect)) k_rec_copy<<<1, 32, 0, c->stream>>>(en4, e0);
        k_rec_row<<<1, 32, 0, c->stream>>>(row, t, cfg->collect, en4, e0, com4);
        if (cfg->collect & ASTER_COLLECT_DISTANCE) {
            const int64_t off = ncol - n;  // the per-body columns come last
            k_rec_distance<<<cgrid, REC_BLOCK, 0, c->stream>>>(n, c->pm.as<double4>(), com4, row + off);
        }
        ASTER_CUDA(cudaGetLastError());
        return ASTER_OK;
    };
    auto advance = [&](int steps) -> int {
        switch (cfg->updater) {
            case ASTER_UPDATER_KDK: return aster_kdk_enqueue(c, p, cfg->solver, cfg->precision, steps);
            case ASTER_UPDATER_SABA:
                return aster_saba_enqueue(c, p, cfg->solver, cfg->precision, cfg->order, steps);
            default: return aster_wh_enqueue(c, p, cfg->precision, steps, m0);
        }
    };
    cudaEventRecord(c->ev[0], c->stream);
    int st = sample(0, 0.0);
    int64_t done = 0;
    for (int64_t k = 1; k < nsamp && st == ASTER_OK; ++k) {
        st = advance(cfg->rate);
        done += cfg->rate;
        if (st == ASTER_OK) st = sample(k, (double)done);
    }
    if (st == ASTER_OK && done < nsteps) st = advance((int)(nsteps - done));  // steps after the last sample
    if (st == ASTER_OK)
        st = cudaMemcpyAsync(rows_out, rows, table * sizeof(double), cudaMemcpyDeviceToHost, c->stream) == cudaSuccess
                 ? ASTER_OK
                 : ASTER_ERR_CUDA;
    cudaEventRecord(c->ev[1], c->stream);
    const int fin = aster_finish(c);
    if (st == ASTER_OK) st = fin;
    if (st != ASTER_OK) c->acc_valid = false;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    return st;
}
