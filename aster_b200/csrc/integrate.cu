// Kick-drift-kick leapfrog driver and FP64 diagnostics.
//
// Replaces update_leapfrog / update_leapfrog_gpu_3d + the `leapfrog` OpenCL
// kernel (src/physics/tool_chain_impl.cpp:169-185, src/utils/updater.cpp:53-87,
// include/Aster/kernels/leapfrog.cl.h:9-29). The reference evaluates the force
// twice per step (before and after the drift); the map it implements is
//   x' = x + v dt + a(x) dt^2/2,  v' = v + (a(x) + a(x')) dt/2,
// which is kick-drift-kick with a(x) reused from the previous step. Here one
// step is two launches:
//   k_kick_drift : v += a dt/2; x += v dt; (mixed: refresh the double-single
//                  copies; LBVH: max |coordinate| for the Morton cube)
//   force kernel : a = A(x) and, fused in its epilogue, v += a dt/2.
// Positions and velocities stay FP64.
//
// Energy replaces Graphs::get_total_energy (src/utils/collectors.cpp:19-53).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "aster_internal.cuh"

namespace {

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <bool MIXED, bool BOX>
__global__ void __launch_bounds__(256) k_kick_drift(int64_t n, double half_dt, double dt,
                                                    double4* __restrict__ pm, double4* __restrict__ vel,
                                                    const double4* __restrict__ acc, float4* __restrict__ phi,
                                                    float4* __restrict__ plo, float4* __restrict__ vf,
                                                    unsigned long long* __restrict__ box_bits) {
    double bmax = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double4 p = pm[i], v = vel[i];
        if (acc) {  // null: drift only (no stale acceleration times zero)
            const double4 a = acc[i];
            v.x += a.x * half_dt; v.y += a.y * half_dt; v.z += a.z * half_dt;
        }
        p.x += v.x * dt; p.y += v.y * dt; p.z += v.z * dt;
        pm[i] = p;
        vel[i] = v;
        if (MIXED) {
            float4 h, l;
            ds_split(p.x, h.x, l.x);
            ds_split(p.y, h.y, l.y);
            ds_split(p.z, h.z, l.z);
            h.w = __double2float_rn(p.w);
            l.w = 0.f;
            phi[i] = h;
            plo[i] = l;
            vf[i] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
        }
        if (BOX) bmax = fmax(bmax, fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))));
    }
    if (BOX) {
        __shared__ double red[8];
        bmax = warp_max(bmax);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = bmax;
        __syncthreads();
        if (threadIdx.x < 32) {
            double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
            v = warp_max(v);
            // non-negative doubles order like their bit patterns
            if (threadIdx.x == 0) atomicMax(box_bits, (unsigned long long)__double_as_longlong(v));
        }
    }
}

// FP64 energy/momentum: per-block partials (ke, pe, px, py, pz), then one
// block adds them in a fixed order (deterministic).
template <bool REF_FORM>
// Block (x, slice y): bodies i of block x against the sources of slice y,
// [y * slice_len, (y + 1) * slice_len); the kinetic energy and momentum of i
// come with slice 0. Partials in part[(y * gridDim.x + x) * 5 + k].
__global__ void __launch_bounds__(256) k_energy_partial(int64_t n, const double4* __restrict__ pm,
                                                        const double4* __restrict__ vel, double eps2,
                                                        int64_t slice_len, double* __restrict__ part) {
    __shared__ double4 sp[256];
    __shared__ double red[5][8];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t j0 = (int64_t)blockIdx.y * slice_len, j1 = min(n, j0 + slice_len);
    double4 pi = i < n ? pm[i] : make_double4(0, 0, 0, 0);
    double pot = 0.0;
    for (int64_t base = j0; base < j1; base += 256) {
        __syncthreads();
        const int64_t j = base + threadIdx.x;
        sp[threadIdx.x] = j < j1 ? pm[j] : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int lim = (int)min((int64_t)256, j1 - base);
        for (int q = 0; q < lim; ++q) {
            if (base + q == i) continue;
            const double4 pj = sp[q];
            double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            double r2 = dx * dx + dy * dy + dz * dz;
            double inv = REF_FORM ? 1.0 / (sqrt(r2) + eps2) : 1.0 / sqrt(r2 + eps2);
            pot += pj.w * inv;
        }
    }
    double v[5] = {0, 0, 0, 0, 0};
    if (i < n) {
        v[1] = -0.5 * pi.w * pot;
        if (blockIdx.y == 0) {
            const double4 vi = vel[i];
            v[0] = 0.5 * pi.w * (vi.x * vi.x + vi.y * vi.y + vi.z * vi.z);
            v[2] = pi.w * vi.x; v[3] = pi.w * vi.y; v[4] = pi.w * vi.z;
        }
    }
    for (int k = 0; k < 5; ++k) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double s = 0;
        for (int w = 0; w < 8; ++w) s += red[threadIdx.x][w];
        part[((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * 5 + threadIdx.x] = s;
    }
}

// out[0] = energy, out[1..3] = momentum from nparts partials: lane l of warp k
// adds component k of partials l, l + 32, ... in order, then a fixed shuffle
// tree (deterministic). 160 threads.
__global__ void __launch_bounds__(160) k_energy_final(int nparts, const double* __restrict__ part, double G,
                                                      double* __restrict__ out) {
    __shared__ double s[5];
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k < 5) {
        double a = 0;
        for (int b = lane; b < nparts; b += 32) a += part[(int64_t)b * 5 + k];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) s[k] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        out[0] = s[0] + G * s[1];
        out[1] = s[2]; out[2] = s[3]; out[3] = s[4];
    }
}

}  // namespace

int aster_kick_drift_launch(aster_ctx* c, const aster_params* p, bool want_box, bool want_mixed) {
    return aster_kick_drift_coef(c, 0.5 * p->dt, p->dt, true, want_box, want_mixed);
}

// v += a * kick_dt (skipped when !kick); x += v * drift_dt.
int aster_kick_drift_coef(aster_ctx* c, double kick_dt, double drift_dt, bool kick, bool want_box, bool want_mixed) {
    c->mixed_valid = want_mixed;  // the kernel refreshes the FP32 copies only when asked
    const int64_t n = c->n;
    int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)c->sm_count * 8);
    if (grid < 1) grid = 1;
    unsigned long long* box = nullptr;
    if (want_box) {
        ASTER_TRY(c->red.ensure(4096));
        box = red_box(c);
        ASTER_CUDA(cudaMemsetAsync(box, 0, sizeof(unsigned long long), c->stream));
    }
    auto* pm = c->pm.as<double4>();
    auto* v = c->vel.as<double4>();
    auto* a = kick ? c->acc.as<double4>() : nullptr;
    const double h = kick_dt, dt = drift_dt;
    if (want_mixed && want_box)
        k_kick_drift<true, true><<<grid, 256, 0, c->stream>>>(n, h, dt, pm, v, a, c->phi.as<float4>(), c->plo.as<float4>(), c->vf.as<float4>(), box);
    else if (want_mixed)
        k_kick_drift<true, false><<<grid, 256, 0, c->stream>>>(n, h, dt, pm, v, a, c->phi.as<float4>(), c->plo.as<float4>(), c->vf.as<float4>(), box);
    else if (want_box)
        k_kick_drift<false, true><<<grid, 256, 0, c->stream>>>(n, h, dt, pm, v, a, nullptr, nullptr, nullptr, box);
    else
        k_kick_drift<false, false><<<grid, 256, 0, c->stream>>>(n, h, dt, pm, v, a, nullptr, nullptr, nullptr, box);
    ASTER_CUDA(cudaGetLastError());
    c->stats.kernels += 1;
    return ASTER_OK;
}

// Per-phase device timing of a time-stepping call: an event pair around every
// build and every force launch, summed after the final synchronisation.
struct PhaseTimer {
    static constexpr int kMax = 2048;
    cudaEvent_t ev[2 * kMax];
    int used = 0;
    bool ok = true;
    ~PhaseTimer() {
        for (int i = 0; i < used; ++i) cudaEventDestroy(ev[i]);
    }
    int fresh() {  // a new event, not recorded; its index, -1 if out of slots
        if (used >= 2 * kMax || cudaEventCreate(&ev[used]) != cudaSuccess) return -1;
        return used++;
    }
    int mark(cudaStream_t s) {  // returns the event index, -1 if out of slots
        if (used >= 2 * kMax || cudaEventCreate(&ev[used]) != cudaSuccess) return -1;
        // under stream capture a plain record only orders streams; External
        // makes it an event-record node of the graph
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(s, &cs);
        if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(ev[used], s, cudaEventRecordExternal);
        else cudaEventRecord(ev[used], s);
        return used++;
    }
    double span(int a, int b) const {
        float ms = 0.f;
        if (a < 0 || b < 0 || cudaEventElapsedTime(&ms, ev[a], ev[b]) != cudaSuccess) return 0.0;
        return ms;
    }
};

static int force_eval(aster_ctx* c, const aster_params* p, int solver, int precision, bool closing_kick,
                      bool box_ready, PhaseTimer* tm, double* ms_build, double* ms_force, int* pairs,
                      bool fuse_next = false) {
    int e0 = tm ? tm->mark(c->stream) : -1;
    if (solver == ASTER_SOLVER_ALLPAIRS) {
        ASTER_TRY(aster_allpairs_launch(c, p, precision, closing_kick, c->n, nullptr, nullptr));
        if (tm) pairs[0] = e0, pairs[1] = e0, pairs[2] = tm->mark(c->stream);
        return ASTER_OK;
    }
    ASTER_TRY(aster_lbvh_build_dev(c, p, box_ready));
    int e1 = tm ? tm->mark(c->stream) : -1;
    ASTER_TRY(aster_lbvh_walk_launch(c, p, precision, closing_kick, nullptr, fuse_next));
    if (tm) pairs[0] = e0, pairs[1] = e1, pairs[2] = tm->mark(c->stream);
    (void)ms_build;
    (void)ms_force;
    return ASTER_OK;
}

// Enqueues step() n times. With graph set, the first step runs as usual
// (allocating whatever a step needs) and the second is captured into a CUDA
// graph that is launched for the remaining n - 1: one launch a step instead of
// one per kernel, which removes the gaps between a step's kernels. The
// captured step's host-side statistics are scaled to n. done() follows every
// step that ran as plain launches; replay(g, ge) precedes every graph launch
// (the timed path re-points the graph's event-record nodes there, so every
// step keeps its own timestamps). Falls back to plain launches when the
// stream cannot be captured (the legacy default stream).
template <class F, class D, class R>
static int repeat_steps(aster_ctx* c, int n, bool graph, F step, D done, R replay) {
    if (n <= 0) return ASTER_OK;
    ASTER_TRY(step());
    ASTER_TRY(done());
    if (n == 1) return ASTER_OK;
    if (graph) {
        const double inter0 = c->stats.interactions;
        const int64_t kern0 = c->stats.kernels;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const int st = step();
            const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            cudaGraphExec_t ge = nullptr;
            if (st == ASTER_OK && e == cudaSuccess && g && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess) {
                c->graphs.push_back({g, ge});
                const double di = c->stats.interactions - inter0;
                const int64_t dk = c->stats.kernels - kern0;
                for (int s = 1; s < n; ++s) {
                    ASTER_TRY(replay(g, ge));
                    ASTER_CUDA(cudaGraphLaunch(ge, c->stream));
                }
                c->stats.interactions += di * (n - 2);
                c->stats.kernels += dk * (n - 2);
                return ASTER_OK;
            }
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();  // the failed capture's error
            if (st != ASTER_OK) return st;
        } else {
            cudaGetLastError();
        }
    }
    for (int s = 1; s < n; ++s) {
        ASTER_TRY(step());
        ASTER_TRY(done());
    }
    return ASTER_OK;
}

static int no_op() { return ASTER_OK; }
static int no_replay(cudaGraph_t, cudaGraphExec_t) { return ASTER_OK; }

// The key of a cached step graph: everything the captured launches depend on
// besides the data in device memory (parameters, solver, precision, body
// count, the addresses of the context's buffers through their generation,
// whether the step carries timing marks).
static std::vector<unsigned char> step_key(const aster_ctx* c, const aster_params* p, int solver, int precision,
                                           bool timed) {
    std::vector<unsigned char> k(sizeof(aster_params));
    std::memcpy(k.data(), p, sizeof(aster_params));
    const int64_t w[] = {solver, precision, timed ? 1 : 0, c->n, c->device, c->walk_stack_limit,
                         (int64_t)aster_devbuf_epoch()};
    const unsigned char* wb = reinterpret_cast<const unsigned char*>(w);
    k.insert(k.end(), wb, wb + sizeof(w));
    return k;
}

// Launches `count` more of the tree KDK's middle step from the context's
// cached graph, capturing it first (one step, `middle`) when the cached one
// does not match this call. The cached graph survives the call, so a later
// call with the same key captures and instantiates nothing: its steps are
// graph launches from the start, and a host thread held up for a few
// milliseconds no longer leaves the GPU idle behind the capture. Without a
// usable graph (capture refused) the steps run as plain launches.
template <class F, class D, class P>
static int middle_graph(aster_ctx* c, const aster_params* p, int solver, int precision, PhaseTimer* tm, int count,
                        F middle, D done, P repoint, const int* last) {
    StepGraph& sg = c->kdk_graph;
    std::vector<unsigned char> key = step_key(c, p, solver, precision, tm != nullptr);
    if (!(sg.ge && sg.key == key)) {
        if (sg.ge) c->graphs.push_back({sg.g, sg.ge});  // may still be queued: destroyed by the next aster_begin
        cudaEvent_t park = sg.park;
        sg = StepGraph{};
        sg.park = park;
        if (!sg.park) ASTER_CUDA(cudaEventCreateWithFlags(&sg.park, cudaEventDisableTiming));
        const double inter0 = c->stats.interactions;
        const int64_t kern0 = c->stats.kernels;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const int st = middle();
            const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            cudaGraphExec_t ge = nullptr;
            if (st == ASTER_OK && e == cudaSuccess && g && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess) {
                sg.g = g;
                sg.ge = ge;
                sg.inter = c->stats.interactions - inter0;
                sg.kernels = c->stats.kernels - kern0;
                c->stats.interactions = inter0;  // counted per launch below
                c->stats.kernels = kern0;
                // every event-record node must be one of this step's marks (re-pointed
                // before each launch) or a context event; otherwise keep it for this call only
                bool keep = true;
                size_t nn = 0;
                ASTER_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
                std::vector<cudaGraphNode_t> nodes(nn);
                ASTER_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
                for (cudaGraphNode_t nd : nodes) {
                    cudaGraphNodeType ty;
                    ASTER_CUDA(cudaGraphNodeGetType(nd, &ty));
                    if (ty != cudaGraphNodeTypeEventRecord && ty != cudaGraphNodeTypeWaitEvent) continue;
                    cudaEvent_t ev = nullptr;
                    if (ty == cudaGraphNodeTypeEventRecord) ASTER_CUDA(cudaGraphEventRecordNodeGetEvent(nd, &ev));
                    else ASTER_CUDA(cudaGraphEventWaitNodeGetEvent(nd, &ev));
                    bool known = false;
                    for (int k = 0; k < 3; ++k)
                        if (tm && last[k] >= 0 && tm->ev[last[k]] == ev && ty == cudaGraphNodeTypeEventRecord) {
                            sg.evnode[k] = nd;
                            known = true;
                        }
                    for (int k = 0; k < 6; ++k)
                        if (c->ev[k] == ev) known = true;
                    keep = keep && known;
                }
                if (keep) sg.key = key;  // an empty key never matches: not reused by a later call
            } else {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();  // the failed capture's error
                if (st != ASTER_OK) return st;
            }
        } else {
            cudaGetLastError();
        }
    }
    int st = ASTER_OK;
    for (int s = 0; s < count && st == ASTER_OK; ++s) {
        bool untimed = false;
        if (sg.ge && tm) st = repoint(sg.ge, sg.evnode, &untimed);
        if (st != ASTER_OK) break;
        if (!sg.ge || untimed) {  // plain launches (their marks, if any, recorded by done)
            st = middle();
            if (st == ASTER_OK) st = done();
            continue;
        }
        const cudaError_t e = cudaGraphLaunch(sg.ge, c->stream);
        if (e != cudaSuccess) st = aster_cuda_fail(e, "cudaGraphLaunch", __FILE__, __LINE__);
        c->stats.interactions += sg.inter;
        c->stats.kernels += sg.kernels;
    }
    // this call's timing events are destroyed when it returns: the marks of the
    // kept graph point at its own event until the next launch re-points them
    // (launches already enqueued keep the events they were launched with)
    if (tm && sg.ge)
        for (int k = 0; k < 3; ++k)
            if (sg.evnode[k]) {
                const cudaError_t e = cudaGraphExecEventRecordNodeSetEvent(sg.ge, sg.evnode[k], sg.park);
                if (e != cudaSuccess && st == ASTER_OK) st = aster_cuda_fail(e, "park", __FILE__, __LINE__);
            }
    return st;
}

// Enqueues nsteps KDK steps (no synchronisation); marks/tm optional.
static int kdk_core(aster_ctx* c, const aster_params* p, int solver, int precision, int nsteps, PhaseTimer* tm,
                    int (*marks)[3], int* nm) {
    const bool mixed_ap = solver == ASTER_SOLVER_ALLPAIRS && precision == ASTER_MIXED;
    int dummy[3];
    if (!c->acc_valid) {
        if (mixed_ap) ASTER_TRY(aster_refresh_mixed(c));
        ASTER_TRY(force_eval(c, p, solver, precision, false, false, tm, nullptr, nullptr, tm ? marks[*nm] : dummy));
        if (tm) ++*nm;
    }
    // the step (kick-drift, force, closing kick) replays as a graph; with phase
    // timing, its three marks are event-record nodes re-pointed before each launch
    int last[3] = {-1, -1, -1};
    cudaGraphNode_t evnode[3] = {nullptr, nullptr, nullptr};
    bool found = false;
    auto step = [&]() -> int {
        ASTER_TRY(aster_kick_drift_launch(c, p, solver == ASTER_SOLVER_LBVH, mixed_ap));
        return force_eval(c, p, solver, precision, true, true, tm, nullptr, nullptr, last);
    };
    // Tree steps: every walk but the last also applies the next step's opening
    // kick and drift (and its bounding box), so only the first step launches
    // the kick-drift kernel: first = kick-drift + build + walk(fused), middle =
    // build + walk(fused) (captured and replayed), last = build + walk.
    const bool fuse = solver == ASTER_SOLVER_LBVH && nsteps >= 2;
    auto first = [&]() -> int {
        ASTER_TRY(aster_kick_drift_launch(c, p, true, false));
        return force_eval(c, p, solver, precision, true, true, tm, nullptr, nullptr, last, true);
    };
    auto middle = [&]() -> int { return force_eval(c, p, solver, precision, true, true, tm, nullptr, nullptr, last, true); };
    auto final_step = [&]() -> int {
        return force_eval(c, p, solver, precision, true, true, tm, nullptr, nullptr, last, false);
    };
    auto done = [&]() -> int {
        if (tm) {
            for (int k = 0; k < 3; ++k) marks[*nm][k] = last[k];
            ++*nm;
        }
        return ASTER_OK;
    };
    // points the step's timing marks (event-record nodes en[]) at fresh events
    // of this call before a launch of ge
    // (*untimed: out of event slots, nothing re-pointed)
    auto repoint = [&](cudaGraphExec_t ge, const cudaGraphNode_t* en, bool* untimed) -> int {
        *untimed = false;
        int m3[3] = {-1, -1, -1};
        for (int k = 0; k < 3; ++k) {
            if (!en[k]) continue;
            // a mark that names the same event as an earlier one (all-pairs: no build span) shares it
            int same = -1;
            for (int q = 0; q < k; ++q)
                if (en[q] == en[k]) same = q;
            if (same >= 0) {
                m3[k] = m3[same];
                continue;
            }
            m3[k] = tm->fresh();
            if (m3[k] < 0) {
                *untimed = true;
                return ASTER_OK;
            }
            ASTER_CUDA(cudaGraphExecEventRecordNodeSetEvent(ge, en[k], tm->ev[m3[k]]));
        }
        for (int k = 0; k < 3; ++k) marks[*nm][k] = m3[k];
        ++*nm;
        return ASTER_OK;
    };
    auto replay = [&](cudaGraph_t g, cudaGraphExec_t ge) -> int {
        if (!tm) return ASTER_OK;
        if (!found) {  // the captured marks' event-record nodes (last[] names the captured events)
            size_t nn = 0;
            ASTER_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
            std::vector<cudaGraphNode_t> nodes(nn);
            ASTER_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
            for (cudaGraphNode_t nd : nodes) {
                cudaGraphNodeType ty;
                ASTER_CUDA(cudaGraphNodeGetType(nd, &ty));
                if (ty != cudaGraphNodeTypeEventRecord) continue;
                cudaEvent_t e = nullptr;
                ASTER_CUDA(cudaGraphEventRecordNodeGetEvent(nd, &e));
                for (int k = 0; k < 3; ++k)
                    if (last[k] >= 0 && tm->ev[last[k]] == e) evnode[k] = nd;
            }
            found = true;
        }
        bool untimed = false;  // out of event slots: the step runs untimed
        return repoint(ge, evnode, &untimed);
    };
    if (fuse) {
        ASTER_TRY(first());
        ASTER_TRY(done());
        const int nmid = nsteps - 2;
        if (nmid > 0) {
            ASTER_TRY(middle());  // plain launches: whatever a step allocates is allocated now
            ASTER_TRY(done());
        }
        if (nmid > 1) ASTER_TRY(middle_graph(c, p, solver, precision, tm, nmid - 1, middle, done, repoint, last));
        ASTER_TRY(final_step());
        ASTER_TRY(done());
    } else {
        ASTER_TRY(repeat_steps(c, nsteps, true, step, done, replay));
    }
    c->acc_valid = true;  // a(x) of the final positions (valid once the work completes without error)
    c->tree.built = false;
    return ASTER_OK;
}

static int kdk_check(aster_ctx* c, const aster_params* p, int solver, int precision, int nsteps) {
    if (!c || nsteps < 0) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    if (solver != ASTER_SOLVER_ALLPAIRS && solver != ASTER_SOLVER_LBVH) return ASTER_ERR_INVALID_ARG;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    return ASTER_OK;
}

int aster_kdk_enqueue(aster_ctx* c, const aster_params* p, int solver, int precision, int nsteps) {
    ASTER_TRY(kdk_check(c, p, solver, precision, nsteps));
    return kdk_core(c, p, solver, precision, nsteps, nullptr, nullptr, nullptr);
}

extern "C" int aster_kdk_steps(aster_ctx* c, const aster_params* p, int solver, int precision, int nsteps) {
    ASTER_TRY(kdk_check(c, p, solver, precision, nsteps));
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    // phase timing (tree path only: build and walk) when the event budget covers every step
    PhaseTimer* tm = solver == ASTER_SOLVER_LBVH && (nsteps + 1) * 3 <= 2 * PhaseTimer::kMax ? new PhaseTimer() : nullptr;
    int marks[3 * (PhaseTimer::kMax / 3 + 2)][3];
    int nm = 0;
    ASTER_TRY(c->red.ensure(4096));
    unsigned long long* inter = red_inter(c);  // walk interaction counter
    ASTER_CUDA(cudaMemsetAsync(inter, 0, sizeof(unsigned long long), c->stream));
    cudaEventRecord(c->ev[0], c->stream);
    int st = kdk_core(c, p, solver, precision, nsteps, tm, marks, &nm);
    if (st != ASTER_OK) {
        delete tm;
        c->acc_valid = false;
        return st;
    }
    cudaEventRecord(c->ev[1], c->stream);
    unsigned long long ic = 0;
    if (solver == ASTER_SOLVER_LBVH)
        ASTER_CUDA(cudaMemcpyAsync(&ic, inter, sizeof(ic), cudaMemcpyDeviceToHost, c->stream));
    st = aster_finish(c);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    if (solver == ASTER_SOLVER_LBVH) c->stats.interactions = (double)ic;
    if (tm) {
        for (int k = 0; k < nm; ++k) {
            c->stats.ms_build += tm->span(marks[k][0], marks[k][1]);
            c->stats.ms_force += tm->span(marks[k][1], marks[k][2]);
        }
        delete tm;
    }
    c->acc_valid = st == ASTER_OK;
    return st;
}

// Host-resident state in, nsteps KDK steps, host state out, in one call: the
// final positions exist after the last step's kick-drift, so their copy to
// the host runs on a second stream while the last force evaluation (tree
// build and walk) runs; velocities and accelerations follow it.
extern "C" int aster_kdk_steps_host(aster_ctx* c, const aster_params* p, int solver, int precision, int nsteps,
                                    int64_t n, double* pos, double* vel, double* acc, const double* mass) {
    if (!c || !pos || !vel || !acc || !mass || n <= 0 || n > (int64_t)1 << 30 || nsteps < 1)
        return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (solver != ASTER_SOLVER_ALLPAIRS && solver != ASTER_SOLVER_LBVH) return ASTER_ERR_INVALID_ARG;
    if (precision != ASTER_FP64 && precision != ASTER_MIXED) return ASTER_ERR_INVALID_ARG;
    if (!c->copy_stream) ASTER_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    cudaEventRecord(c->ev[0], c->stream);
    // the tree path reads no mass before its build: their copy overlaps the first kick-drift and sort
    // one tree step: its opening kick and drift are applied while the state is unpacked
    const bool fused = solver == ASTER_SOLVER_LBVH && nsteps == 1;
    int st = solver == ASTER_SOLVER_LBVH ? aster_upload_enqueue_overlapped(c, n, pos, vel, mass, acc, fused ? p : nullptr)
                                         : aster_upload_enqueue(c, n, pos, vel, mass, acc);
    const bool mixed_ap = solver == ASTER_SOLVER_ALLPAIRS && precision == ASTER_MIXED;
    int dummy[3];
    if (st == ASTER_OK && nsteps > 1) st = kdk_core(c, p, solver, precision, nsteps - 1, nullptr, nullptr, nullptr);
    if (st == ASTER_OK && !fused) st = aster_kick_drift_launch(c, p, solver == ASTER_SOLVER_LBVH, mixed_ap);
    if (st == ASTER_OK) {
        // positions are final: copy them out on the second stream
        cudaEventRecord(c->ev[2], c->stream);
        ASTER_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev[2], 0));
        st = aster_download_enqueue(c, 0, pos, c->copy_stream);
    }
    if (st == ASTER_OK) st = force_eval(c, p, solver, precision, true, true, nullptr, nullptr, nullptr, dummy);
    if (st == ASTER_OK) st = aster_download_va_enqueue(c, vel, acc, c->stream);
    cudaEventRecord(c->ev[1], c->stream);
    const cudaError_t ce = cudaStreamSynchronize(c->copy_stream);
    const int fin = aster_finish(c);
    if (st == ASTER_OK && ce != cudaSuccess) st = aster_cuda_fail(ce, "cudaStreamSynchronize", __FILE__, __LINE__);
    if (st == ASTER_OK) st = fin;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->acc_valid = st == ASTER_OK;
    c->tree.built = false;
    c->mass_pending = nullptr;  // consumed by the build, or void after an error
    if (st != ASTER_OK) c->n = 0;  // the resident state is not trustworthy after a failed upload or step
    return st;
}

// SABA_n drift/kick coefficients (Laskar & Robutel 2001): with x_1 < ... < x_n
// the Gauss-Legendre nodes on [0,1] and w_k the weights, the drifts are
// c_1 = x_1, c_{k+1} = x_{k+1} - x_k, c_{n+1} = 1 - x_n and the kicks d_k = w_k
// (the values include/Aster/physics/coeffs.h:8-161 tabulates, there to 35
// digits). Nodes by Newton's method on the Legendre three-term recurrence in
// long double, then rounded once. Returns the number of kicks.
static int saba_coeffs(int order, double* c, double* d) {
    const int n = order;
    long double x[10] = {0}, w[10] = {0};
    const long double pi = 3.141592653589793238462643383279502884L;
    auto legendre = [n](long double z, long double& dp) {
        long double p0 = 1.0L, p1 = z;
        for (int k = 2; k <= n; ++k) {
            const long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0L);
        return p1;
    };
    for (int i = 0; i < n; ++i) {
        long double z = std::cos(pi * (i + 0.75L) / (n + 0.5L)), dp = 1.0L;
        for (int it = 0; it < 100; ++it) {
            const long double dz = legendre(z, dp) / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-19L) break;
        }
        legendre(z, dp);
        x[n - 1 - i] = 0.5L * (1.0L + z);  // ascending on [0,1]
        w[n - 1 - i] = 1.0L / ((1.0L - z * z) * dp * dp);
    }
    c[0] = (double)x[0];
    for (int k = 1; k < n; ++k) c[k] = (double)(x[k] - x[k - 1]);
    c[n] = (double)(1.0L - x[n - 1]);
    for (int k = 0; k < n; ++k) d[k] = (double)w[k];
    return n;
}

// Enqueues nsteps SABA_order steps (no synchronisation).
static int saba_core(aster_ctx* c, const aster_params* p, int solver, int precision, int order, int nsteps,
                     PhaseTimer* tm, std::vector<std::array<int, 3>>* marks) {
    double cc[11], dd[10];
    int nk = 1;
    if (order > 1) nk = saba_coeffs(order, cc, dd);
    const bool lbvh = solver == ASTER_SOLVER_LBVH;
    const bool mixed_ap = solver == ASTER_SOLVER_ALLPAIRS && precision == ASTER_MIXED;
    auto force = [&](bool box_ready) -> int {
        int m3[3] = {-1, -1, -1};
        ASTER_TRY(force_eval(c, p, solver, precision, false, box_ready, tm, nullptr, nullptr, m3));
        if (tm) marks->push_back({m3[0], m3[1], m3[2]});
        return ASTER_OK;
    };
    const double dt = p->dt;
    if (order == 1 && mixed_ap) ASTER_TRY(aster_refresh_mixed(c));
    if (order == 1 && nsteps > 0) {
        ASTER_TRY(force(false));  // the first Euler step computes its own box
        ASTER_TRY(aster_kick_drift_coef(c, dt, dt, true, lbvh, mixed_ap));
        --nsteps;
    }
    // the all-pairs step replays as a graph
    ASTER_TRY(repeat_steps(c, nsteps, !lbvh && !tm, [&]() -> int {
        if (order == 1) {
            ASTER_TRY(force(true));
            return aster_kick_drift_coef(c, dt, dt, true, lbvh, mixed_ap);
        }
        ASTER_TRY(aster_kick_drift_coef(c, 0.0, cc[0] * dt, false, lbvh, mixed_ap));
        for (int k = 0; k < nk; ++k) {
            ASTER_TRY(force(true));
            ASTER_TRY(aster_kick_drift_coef(c, dd[k] * dt, cc[k + 1] * dt, true, lbvh, mixed_ap));
        }
        return ASTER_OK;
    }, no_op, no_replay));
    c->acc_valid = false;  // the last drift moved the bodies after the last force evaluation
    c->tree.built = false;
    return ASTER_OK;
}

static int saba_check(aster_ctx* c, const aster_params* p, int solver, int precision, int order, int nsteps) {
    if (!c || nsteps < 0 || order < 1 || order > 10) return ASTER_ERR_INVALID_ARG;
    return kdk_check(c, p, solver, precision, nsteps);
}

int aster_saba_enqueue(aster_ctx* c, const aster_params* p, int solver, int precision, int order, int nsteps) {
    ASTER_TRY(saba_check(c, p, solver, precision, order, nsteps));
    return saba_core(c, p, solver, precision, order, nsteps, nullptr, nullptr);
}

// Replaces update_SABA1..10 (src/integrators/SABA.cpp:14-553) and the OpenCL
// SABA updater (src/utils/tc_impl_cl.cpp:269-299 + generalized_intgrt3d.cl.h).
// Order n >= 2, per step: drift c_1; then n times: forces, kick d_k and drift
// c_{k+1} in one launch. Order 1 is the reference's SABA1 = update_euler:
// forces, v += a dt, x += v dt. Differences from the reference, on purpose:
// its OpenCL updater binds d to the kernel's c argument and c to d (the kick
// uses the drift coefficient and vice versa) and evaluates the forces twice
// per slot; its CPU update_SABA6 kicks with d2 where the sequence (and its own
// coefficient table) has d3. Here every order follows the published sequence.
extern "C" int aster_saba_steps(aster_ctx* c, const aster_params* p, int solver, int precision, int order,
                                int nsteps) {
    ASTER_TRY(saba_check(c, p, solver, precision, order, nsteps));
    ASTER_TRY(aster_begin(c));
    c->stats = aster_stats{};
    const bool lbvh = solver == ASTER_SOLVER_LBVH;
    const int nk = order > 1 ? order : 1;
    PhaseTimer* tm = lbvh && (int64_t)(nsteps * nk + 1) * 3 <= 2 * PhaseTimer::kMax ? new PhaseTimer() : nullptr;
    std::vector<std::array<int, 3>> marks;
    ASTER_TRY(c->red.ensure(4096));
    unsigned long long* inter = red_inter(c);
    ASTER_CUDA(cudaMemsetAsync(inter, 0, sizeof(unsigned long long), c->stream));
    cudaEventRecord(c->ev[0], c->stream);
    int st = saba_core(c, p, solver, precision, order, nsteps, tm, &marks);
    if (st != ASTER_OK) {
        delete tm;
        return st;
    }
    cudaEventRecord(c->ev[1], c->stream);
    unsigned long long ic = 0;
    if (lbvh) ASTER_CUDA(cudaMemcpyAsync(&ic, inter, sizeof(ic), cudaMemcpyDeviceToHost, c->stream));
    st = aster_finish(c);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    if (lbvh) c->stats.interactions = (double)ic;
    if (tm) {
        for (const auto& m3 : marks) {
            c->stats.ms_build += tm->span(m3[0], m3[1]);
            c->stats.ms_force += tm->span(m3[1], m3[2]);
        }
        delete tm;
    }
    return st;
}

// FP64 energy and momentum of the resident state into out4 (device:
// energy, px, py, pz); part holds (n + 255) / 256 * 5 doubles. No sync.
// Source slices of the energy sum: enough blocks to fill the GPU when n is
// small (each slice a whole number of 256-body tiles).
static int energy_slices(const aster_ctx* c, int64_t n) {
    const int64_t tiles = (n + 255) / 256;
    int64_t ns = ((int64_t)4 * c->sm_count + tiles - 1) / tiles;
    if (ns > tiles) ns = tiles;
    if (ns > 64) ns = 64;
    if (ns < 1) ns = 1;
    return (int)ns;
}

// Partials (5 doubles each) that aster_energy_enqueue writes.
int64_t aster_energy_parts(const aster_ctx* c) { return (c->n + 255) / 256 * energy_slices(c, c->n); }

int aster_energy_enqueue(aster_ctx* c, const aster_params* p, int ref_form, double* part, double* out4) {
    const int64_t n = c->n;
    const int nb = (int)((n + 255) / 256);
    const int ns = energy_slices(c, n);
    const int64_t slice_len = (nb + ns - 1) / ns * (int64_t)256;
    const dim3 grid((unsigned)nb, (unsigned)ns);
    if (ref_form)
        k_energy_partial<true><<<grid, 256, 0, c->stream>>>(n, c->pm.as<double4>(), c->vel.as<double4>(), p->eps2,
                                                            slice_len, part);
    else
        k_energy_partial<false><<<grid, 256, 0, c->stream>>>(n, c->pm.as<double4>(), c->vel.as<double4>(), p->eps2,
                                                             slice_len, part);
    ASTER_CUDA(cudaGetLastError());
    k_energy_final<<<1, 160, 0, c->stream>>>(nb * ns, part, p->G, out4);
    ASTER_CUDA(cudaGetLastError());
    return ASTER_OK;
}

extern "C" int aster_energy(aster_ctx* c, const aster_params* p, int ref_form, double* energy, double* momentum3) {
    if (!c || !energy) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    ASTER_TRY(aster_begin(c));
    ASTER_TRY(c->scratch.ensure((size_t)aster_energy_parts(c) * 5 * sizeof(double) + 64));
    ASTER_TRY(c->red.ensure(4096));
    double* part = c->scratch.as<double>();
    double* out = red_energy(c);
    ASTER_TRY(aster_energy_enqueue(c, p, ref_form, part, out));
    double host[4];
    ASTER_CUDA(cudaMemcpyAsync(host, out, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    ASTER_TRY(aster_finish(c));
    *energy = host[0];
    if (momentum3) { momentum3[0] = host[1]; momentum3[1] = host[2]; momentum3[2] = host[3]; }
    return ASTER_OK;
}

// ---- allocation-free energy ------------------------------------------------
// aster_energy_noalloc runs the same two kernels as aster_energy but keeps the
// per-block partial sums (5 doubles per 256 bodies) in the file-scope device
// array below instead of context memory, so the call allocates nothing. The
// array is part of the module: every GPU that loads this library holds it
// (ASTER_ENERGY_NOALLOC_MAX_N / 256 * 5 doubles = 2.5 MiB) until the process
// exits. Device code could name the array directly; host code must not pass
// &g_energy_partials to a kernel (on the host that name is only a stand-in),
// so each device's address is fetched once with cudaGetSymbolAddress and kept.
static constexpr int64_t kEnergyNoAllocMaxBlocks = ASTER_ENERGY_NOALLOC_MAX_N / 256;
static constexpr int kEnergyNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_energy_partials[kEnergyNoAllocMaxBlocks * 5];
static double* g_energy_partials_addr[kEnergyNoAllocMaxDevices];
static std::mutex g_energy_partials_mu;

// Address of g_energy_partials on the current device; the first call on a
// device looks it up (with that device current) and caches it.
static int energy_partials_on_current_device(double** out) {
    int dev = -1;
    ASTER_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kEnergyNoAllocMaxDevices) return ASTER_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_energy_partials_mu);
    if (!g_energy_partials_addr[dev]) {
        void* ptr = nullptr;
        ASTER_CUDA(cudaGetSymbolAddress(&ptr, g_energy_partials));
        g_energy_partials_addr[dev] = static_cast<double*>(ptr);
    }
    *out = g_energy_partials_addr[dev];
    return ASTER_OK;
}

extern "C" int aster_energy_noalloc(int64_t n, const double* pm_dev, const double* vel_dev, const aster_params* p,
                                    int ref_form, double* out_dev, void* stream) {
    if (n <= 0 || !pm_dev || !vel_dev || !out_dev) return ASTER_ERR_INVALID_ARG;
    if (((uintptr_t)pm_dev & 31) || ((uintptr_t)vel_dev & 31) || ((uintptr_t)out_dev & 7))
        return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_check_params(p));
    if (n > ASTER_ENERGY_NOALLOC_MAX_N) return ASTER_ERR_TOO_LARGE;
    const int nb = (int)((n + 255) / 256);
    double* part = nullptr;
    ASTER_TRY(energy_partials_on_current_device(&part));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double4* pm = reinterpret_cast<const double4*>(pm_dev);
    const double4* vel = reinterpret_cast<const double4*>(vel_dev);
    const int64_t whole = (int64_t)nb * 256;  // one slice: every source
    if (ref_form)
        k_energy_partial<true><<<nb, 256, 0, st>>>(n, pm, vel, p->eps2, whole, part);
    else
        k_energy_partial<false><<<nb, 256, 0, st>>>(n, pm, vel, p->eps2, whole, part);
    ASTER_CUDA(cudaGetLastError());
    k_energy_final<<<1, 160, 0, st>>>(nb, part, p->G, out_dev);
    ASTER_CUDA(cudaGetLastError());
    return ASTER_OK;
}
