// Internal declarations shared by the CUDA translation units of
// libaster_cuda.so. Not part of the C ABI (include/aster_cuda.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <utility>
#include <vector>

#include "../../include/aster_cuda.h"

// Device error flag bits (ctx->err_dev). Kernels OR a bit in and stop the
// affected work; the host turns the first bit found into a status code.
#define ASTER_DEVERR_STACK 0x1
#define ASTER_DEVERR_TREE 0x2
#define ASTER_DEVERR_NONFINITE 0x4
#define ASTER_DEVERR_CANCEL 0x8
#define ASTER_DEVERR_LIST 0x10
#define ASTER_DEVERR_KEPLER 0x20

// The O(N^2) kernels (all-pairs forces, adjoint pair terms) split the sources
// into slices when there are too few target blocks to give every SM this many
// blocks (small N), and add the slices' partial sums afterwards. Measured
// (same-box A/B, 2 / 4 / 6 / 8 / 12): 12 took the C5 adjoint (N = 16384,
// 1000 steps) from 1021 to 744 ms mixed and 2057 to 1400 ms FP64, and the C1
// FP64 step (N = 4096) from 0.048 to 0.040 ms. The mixed all-pairs kernel
// keeps at least ASTER_SLICE_MIN_MIXED sources per slice: with 128 the C1
// mixed step slowed from 0.0255 to 0.0274 ms, the reduction of 32 partial
// sums per body outweighing the parallelism.
#ifndef ASTER_SLICE_BLOCKS_PER_SM
#define ASTER_SLICE_BLOCKS_PER_SM 12
#endif
#ifndef ASTER_SLICE_MIN_MIXED
#define ASTER_SLICE_MIN_MIXED 256
#endif

#define ASTER_TRY(...)                                    \
    do {                                                  \
        int _st = (__VA_ARGS__);                          \
        if (_st != ASTER_OK) return _st;                  \
    } while (0)

#define ASTER_CUDA(expr)                                  \
    do {                                                  \
        cudaError_t _e = (expr);                          \
        if (_e != cudaSuccess) return aster_cuda_fail(_e, #expr, __FILE__, __LINE__); \
    } while (0)

int aster_cuda_fail(cudaError_t e, const char* what, const char* file, int line);

// Generation of the device buffers: changes whenever any DevBuf is allocated
// or freed, so that a cached graph (which holds buffer addresses) is only
// replayed while every buffer it names still lives where it was captured.
unsigned long long aster_devbuf_epoch();

// Grow-only device buffer.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t want);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// LBVH device arrays (sized for n bodies, 2n-1 nodes).
struct LbvhBufs {
    DevBuf codes, codes_alt, sorted_codes, perm, perm_alt, hist, digit_off;
    DevBuf parent, sib, rlo, rhi, counters;
    DevBuf node_cm, bmin, bmax;  // node_cm: double4 (com x, y, z, mass)
    DevBuf child, groups, crec, front;
    DevBuf node_v;  // double4 (vx, vy, vz, 0) per node: post-Newtonian walk only
    int64_t n = 0;
    bool built = false;
    double box = 0.0;
};

// Batched-ensemble device arrays.
struct EnsBufs {
    DevBuf pm, vel, off, order, counter;
    int32_t nsys = 0;
    int64_t nbodies = 0;
    double pair_evals_per_stage = 0.0;   // sum over systems of n(n-1)
    volatile int* cancel_host = nullptr;  // pinned, mapped
    int* cancel_dev = nullptr;
};

// Adjoint (reverse-mode) buffers.
struct AdjBufs {
    DevBuf ckpt, segx, lx, lv, lm, w, target, part;
};

// An executable graph of one repeated step, kept across calls: replayed by
// a later call whose key (parameters, sizes, buffer generation, timing on or
// off) is the same, so that call captures and instantiates nothing.
struct StepGraph {
    std::vector<unsigned char> key;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    cudaGraphNode_t evnode[3] = {nullptr, nullptr, nullptr};  // the step's timing marks (re-pointed per launch)
    // between calls the marks point here (the events of a call's timing die
    // with the call; an executable graph must not keep naming them)
    cudaEvent_t park = nullptr;
    double inter = 0.0;                                         // host-side counts of one step
    int64_t kernels = 0;
};

struct aster_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t copy_stream = nullptr;  // device->host copies overlapped with compute (created on first use)
    int64_t n = 0;
    int64_t n_src = 0;  // 1 + index of the last body with non-zero mass: all-pairs sources stop there
    DevBuf pm;    // double4 (x, y, z, m), input order
    DevBuf vel;   // double4 (vx, vy, vz, 0)
    DevBuf acc;   // double4 (ax, ay, az, 0): cached acceleration
    DevBuf phi;   // float4 (x_hi, y_hi, z_hi, m): round-to-nearest of x
    DevBuf plo;   // float4 (x - x_hi, ..., 0): double-single low parts
    DevBuf vf;    // float4 (vx, vy, vz, 0) for PN terms in FP32
    DevBuf scratch;   // j-split partial accumulators, reductions
    DevBuf targets;   // target list for aster_allpairs_targets
    DevBuf stage;     // device staging for AoS <-> SoA-4 conversion
    DevBuf red;       // small reduction buffers (box, energy)
    DevBuf wh;        // Wisdom-Holman: reduction partials and state scalars
    DevBuf rec;       // aster_record: the sample table and its reductions
    bool acc_valid = false;
    // phi/plo/vf (the FP32 copies the mixed all-pairs kernels read) match
    // pm/vel; anything that moves positions or velocities without refreshing
    // them clears it, and a mixed all-pairs launch refreshes them first
    bool mixed_valid = false;
    int* err_dev = nullptr;     // device error flags
    int* err_host = nullptr;    // pinned copy
    int* stack_hw_dev = nullptr;  // tree-walk stack high-water mark
    // usable tree-walk stack entries per warp (<= the 1024 in shared memory);
    // ASTER_WALK_STACK_LIMIT lowers it, e.g. to exercise the overflow path
    int walk_stack_limit = 1024;
    LbvhBufs tree;
    EnsBufs ens;
    AdjBufs adj;
    aster_stats stats{};
    // [0], [1] timing; [2] final positions ready; [3] upload copies issued;
    // [4] masses copied (overlapped upload)
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    // masses still on their way (overlapped upload): staging copy on the
    // device, applied to pm[].w before the tree build reads them
    const double* mass_pending = nullptr;
    // executable graphs of the last call's repeated steps; destroyed by the
    // next call's aster_begin (its work has finished by then) or at destroy
    std::vector<std::pair<cudaGraph_t, cudaGraphExec_t>> graphs;
    // the tree KDK's middle step (kick-fused build + walk), kept across calls;
    // a replaced one moves to `graphs`
    StepGraph kdk_graph;
};

// Layout of ctx->red (4 KB of small device scalars).
inline unsigned long long* red_box(aster_ctx* c) { return c->red.as<unsigned long long>(); }         // byte 0
inline double* red_energy(aster_ctx* c) { return c->red.as<double>() + 8; }                         // byte 64
inline unsigned long long* red_inter(aster_ctx* c) { return c->red.as<unsigned long long>() + 64; } // byte 512
inline unsigned int* red_groups(aster_ctx* c) {  // [0] large-group count, [1] walk work counter, [2] bottom-up
                                                 // frontier, [3] small-group count
    return reinterpret_cast<unsigned int*>(c->red.as<char>() + 1024);
}

// ---- shared host helpers (context.cu) -------------------------------------
int aster_check_params(const aster_params* p);
int aster_begin(aster_ctx* ctx);                // clears the device error flag
int aster_finish(aster_ctx* ctx);               // syncs, turns flags into status
int aster_refresh_mixed(aster_ctx* ctx);        // rebuild phi/plo/vf from pm/vel
// Host state -> device with the masses' copy overlapped (see context.cu); with
// kick_drift, the first KDK step's opening kick, drift and bounding box
// (red_box) are applied while unpacking, so its kick-drift launch is left out
int aster_upload_enqueue_overlapped(aster_ctx* c, int64_t n, const double* pos, const double* vel, const double* mass,
                                    const double* acc, const aster_params* kick_drift = nullptr);
// velocities and accelerations -> host (one unpack, two back-to-back copies)
int aster_download_va_enqueue(aster_ctx* c, double* vel, double* acc, cudaStream_t stream);
// applies masses still on their way (waits for their copy); no-op otherwise
int aster_apply_pending_mass(aster_ctx* c);
int aster_copy_acc_out(aster_ctx* ctx, double* acc_out);

// ---- kernels exposed across translation units ------------------------------
// allpairs.cu
int aster_allpairs_launch(aster_ctx* ctx, const aster_params* p, int precision,
                          bool closing_kick, int64_t nt, const int32_t* targets_dev,
                          double* out_dev /* nt*3 or null: write ctx->acc */);
int aster_allpairs_launch_range(aster_ctx* ctx, const aster_params* p, int precision, bool closing_kick, int64_t nt,
                                const int32_t* targets_dev, double* out_dev, int64_t src_lo, int64_t src_hi);
// integrate.cu
int aster_kick_drift_launch(aster_ctx* ctx, const aster_params* p, bool want_box, bool want_mixed);
// Enqueue-only cores of the stepping entry points (argument checks included,
// no synchronisation): used by aster_record to step and sample on the device.
int aster_kdk_enqueue(aster_ctx* ctx, const aster_params* p, int solver, int precision, int nsteps);
int aster_saba_enqueue(aster_ctx* ctx, const aster_params* p, int solver, int precision, int order, int nsteps);
int aster_wh_central_mass(aster_ctx* ctx, double* m0);  // synchronises; ASTER_ERR_INVALID_ARG if <= 0
int aster_wh_enqueue(aster_ctx* ctx, const aster_params* p, int precision, int nsteps, double m0);
// host state -> device on the context stream (no synchronisation; arguments
// checked by the caller); acc (optional) becomes the cached acceleration
int aster_upload_enqueue(aster_ctx* ctx, int64_t n, const double* pos, const double* vel, const double* mass,
                         const double* acc);
// state array `which` (0 positions, 1 velocities, 2 accelerations) -> host on `stream`
int aster_download_enqueue(aster_ctx* ctx, int which, double* host, cudaStream_t stream);
// energy and momentum into out4 (device); part: aster_energy_parts(ctx) * 5 doubles
int aster_energy_enqueue(aster_ctx* ctx, const aster_params* p, int ref_form, double* part, double* out4);
int64_t aster_energy_parts(const aster_ctx* ctx);
// v += a * kick_dt (skipped when !kick), x += v * drift_dt, refresh derived copies
int aster_kick_drift_coef(aster_ctx* ctx, double kick_dt, double drift_dt, bool kick, bool want_box,
                          bool want_mixed);
// lbvh.cu
int aster_lbvh_build_dev(aster_ctx* ctx, const aster_params* p, bool box_ready);
// fuse_next (with closing_kick): the walk also applies the next step's
// opening kick and drift to every body and leaves their bounding box in
// red_box, so that step's kick-drift launch is left out.
int aster_lbvh_walk_launch(aster_ctx* ctx, const aster_params* p, int precision,
                           bool closing_kick, int32_t* list_counts_dev, bool fuse_next = false);

// ---- device helpers --------------------------------------------------------
__device__ __forceinline__ void ds_split(double x, float& hi, float& lo) {
    hi = __double2float_rn(x);
    lo = __double2float_rn(__dsub_rn(x, (double)hi));
}

// Error-free transformation a + b = s + e (Knuth two-sum, FP32), written with
// explicitly rounded intrinsics so that no FMA contraction can cancel it.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    float bp = __fsub_rn(s, a);
    float ap = __fsub_rn(s, bp);
    e = __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp));
}

// Compensated accumulator: value = hi + lo. add() folds one FP32 partial in.
struct CompSum {
    float hi = 0.f, lo = 0.f;
    __device__ __forceinline__ void add(float x) {
        float s, e;
        two_sum(hi, x, s, e);
        hi = s;
        lo = __fadd_rn(lo, e);
    }
    __device__ __forceinline__ double value() const { return (double)hi + (double)lo; }
};

__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
