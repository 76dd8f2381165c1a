// Context, state transfer, error handling and the shared host helpers of the
// C ABI (include/aster_cuda.h). The state upload/download replace the
// reference's Simulation::load_gpu_buffers / read_bodies_gpu
// (src/utils/builder_endpoint.cpp:102-119, 424-434): the reference copies
// std::vector<vec3> (AoS FP64) into OpenCL buffers; here AoS FP64 host arrays
// are packed into 32-byte double4 records (x, y, z, m) and (vx, vy, vz, 0) so
// that every body is one aligned 32-byte load.
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>

#include "aster_internal.cuh"

static thread_local char g_last_error[256] = "";
static void release_graphs(aster_ctx* c);

int aster_cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    return e == cudaErrorMemoryAllocation ? ASTER_ERR_OOM : ASTER_ERR_CUDA;
}

static std::atomic<unsigned long long> g_devbuf_epoch{0};
unsigned long long aster_devbuf_epoch() { return g_devbuf_epoch.load(); }

int DevBuf::ensure(size_t want) {
    if (want <= bytes && ptr) return ASTER_OK;
    release();
    size_t b = want < 256 ? 256 : want;
    ++g_devbuf_epoch;
    cudaError_t e = cudaMalloc(&ptr, b);
    if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        cudaGetLastError();
        return aster_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    }
    bytes = b;
    return ASTER_OK;
}

void DevBuf::release() {
    if (ptr) {
        ++g_devbuf_epoch;
        cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
}

extern "C" const char* aster_strerror(int s) {
    switch (s) {
        case ASTER_OK: return "ok";
        case ASTER_ERR_INVALID_ARG: return "invalid argument";
        case ASTER_ERR_CUDA: return g_last_error[0] ? g_last_error : "CUDA runtime error";
        case ASTER_ERR_OOM: return "device out of memory";
        case ASTER_ERR_NO_STATE: return "no body state uploaded";
        case ASTER_ERR_STACK: return "tree-walk stack overflow";
        case ASTER_ERR_TREE: return "bottom-up climb exceeded level cap";
        case ASTER_ERR_NONFINITE: return "non-finite value in state or result";
        case ASTER_ERR_CANCELLED: return "cancelled";
        case ASTER_ERR_UNSUPPORTED: return "unsupported option";
        case ASTER_ERR_TOO_LARGE: return "size beyond fixed capacity";
        case ASTER_ERR_KEPLER: return "Kepler drift did not converge (or a body sits on the central mass)";
        default: return "unknown status";
    }
}

extern "C" int aster_version(void) { return 10000; }

int aster_check_params(const aster_params* p) {
    if (!p) return ASTER_ERR_INVALID_ARG;
    if (!std::isfinite(p->G) || !std::isfinite(p->eps2) || p->eps2 < 0.0) return ASTER_ERR_INVALID_ARG;
    if (!std::isfinite(p->dt) || !std::isfinite(p->theta) || p->theta < 0.0) return ASTER_ERR_INVALID_ARG;
    const int32_t pn_bits = ASTER_PN1 | ASTER_PN2 | ASTER_PN25;
    if ((p->force_law & pn_bits) && !(std::isfinite(p->c) && p->c > 0.0)) return ASTER_ERR_INVALID_ARG;
    if (p->force_law & ~(ASTER_NEWTON | pn_bits)) return ASTER_ERR_UNSUPPORTED;
    if (p->morton_bits != 30 && p->morton_bits != 63) return ASTER_ERR_INVALID_ARG;
    if (p->compat_mode != 0 && p->compat_mode != 1) return ASTER_ERR_INVALID_ARG;
    if (p->compat_mode == 1 && p->morton_bits != 30) return ASTER_ERR_UNSUPPORTED;
    if (p->reserved != 0) return ASTER_ERR_INVALID_ARG;
    return ASTER_OK;
}

extern "C" int aster_ctx_create(aster_ctx** out, int device, void* stream) {
    if (!out) return ASTER_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    ASTER_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return ASTER_ERR_INVALID_ARG;
    ASTER_CUDA(cudaSetDevice(device));
    aster_ctx* c = new (std::nothrow) aster_ctx();
    if (!c) return ASTER_ERR_OOM;
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete c; return aster_cuda_fail(e, "cudaStreamCreate", __FILE__, __LINE__); }
        c->own_stream = true;
    }
    cudaError_t e = cudaMalloc(&c->err_dev, 2 * sizeof(int));
    if (e == cudaSuccess) e = cudaHostAlloc(&c->err_host, 2 * sizeof(int), cudaHostAllocDefault);
    for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&c->ev[i]);
    if (e != cudaSuccess) {
        aster_ctx_destroy(c);
        return aster_cuda_fail(e, "aster_ctx_create", __FILE__, __LINE__);
    }
    c->stack_hw_dev = c->err_dev + 1;
    if (const char* lim = std::getenv("ASTER_WALK_STACK_LIMIT")) {
        const int v = std::atoi(lim);
        if (v >= 64 && v < c->walk_stack_limit) c->walk_stack_limit = v;
    }
    cudaMemset(c->err_dev, 0, 2 * sizeof(int));
    *out = c;
    return ASTER_OK;
}

extern "C" int aster_ctx_destroy(aster_ctx* c) {
    if (!c) return ASTER_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    release_graphs(c);
    if (c->kdk_graph.ge) cudaGraphExecDestroy(c->kdk_graph.ge);
    if (c->kdk_graph.g) cudaGraphDestroy(c->kdk_graph.g);
    if (c->kdk_graph.park) cudaEventDestroy(c->kdk_graph.park);
    DevBuf* bufs[] = {&c->pm, &c->vel, &c->acc, &c->phi, &c->plo, &c->vf, &c->scratch, &c->targets,
                      &c->stage, &c->red, &c->wh, &c->rec,
                      &c->tree.codes, &c->tree.codes_alt, &c->tree.sorted_codes, &c->tree.perm,
                      &c->tree.perm_alt, &c->tree.hist, &c->tree.digit_off,
                      &c->tree.parent, &c->tree.sib, &c->tree.rlo, &c->tree.rhi, &c->tree.counters, &c->tree.node_cm,
                      &c->tree.bmin, &c->tree.bmax, &c->tree.child, &c->tree.groups, &c->tree.crec, &c->tree.front,
                      &c->tree.node_v};
    for (DevBuf* b : bufs) b->release();
    DevBuf* ens[] = {&c->ens.pm, &c->ens.vel, &c->ens.off, &c->ens.order, &c->ens.counter,
                     &c->adj.ckpt, &c->adj.segx, &c->adj.lx, &c->adj.lv, &c->adj.lm, &c->adj.w,
                     &c->adj.target, &c->adj.part};
    for (DevBuf* b : ens) b->release();
    if (c->ens.cancel_host) cudaFreeHost((void*)c->ens.cancel_host);
    for (int i = 0; i < 6; ++i)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    if (c->err_dev) cudaFree(c->err_dev);
    if (c->err_host) cudaFreeHost(c->err_host);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    delete c;
    return ASTER_OK;
}

static void release_graphs(aster_ctx* c) {
    for (auto& g : c->graphs) {
        if (g.second) cudaGraphExecDestroy(g.second);
        if (g.first) cudaGraphDestroy(g.first);
    }
    c->graphs.clear();
}

int aster_begin(aster_ctx* c) {
    ASTER_CUDA(cudaSetDevice(c->device));
    release_graphs(c);  // the previous call synchronised before returning
    ASTER_CUDA(cudaMemsetAsync(c->err_dev, 0, 2 * sizeof(int), c->stream));
    return ASTER_OK;
}

int aster_finish(aster_ctx* c) {
    ASTER_CUDA(cudaMemcpyAsync(c->err_host, c->err_dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    ASTER_CUDA(cudaStreamSynchronize(c->stream));
    ASTER_CUDA(cudaGetLastError());
    int f = c->err_host[0];
    c->stats.max_stack = c->err_host[1];
    if (f & ASTER_DEVERR_STACK) return ASTER_ERR_STACK;
    if (f & ASTER_DEVERR_LIST) return ASTER_ERR_STACK;
    if (f & ASTER_DEVERR_TREE) return ASTER_ERR_TREE;
    if (f & ASTER_DEVERR_CANCEL) return ASTER_ERR_CANCELLED;
    if (f & ASTER_DEVERR_NONFINITE) return ASTER_ERR_NONFINITE;
    if (f & ASTER_DEVERR_KEPLER) return ASTER_ERR_KEPLER;
    return ASTER_OK;
}

// ---- packing kernels --------------------------------------------------------
__global__ void k_pack_state(int64_t n, const double* __restrict__ pos, const double* __restrict__ vel,
                             const double* __restrict__ mass, double4* __restrict__ pm,
                             double4* __restrict__ v4, float4* __restrict__ phi,
                             float4* __restrict__ plo, float4* __restrict__ vf, int* err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2], m = mass[i];
        double vx = 0, vy = 0, vz = 0;
        if (vel) { vx = vel[3 * i]; vy = vel[3 * i + 1]; vz = vel[3 * i + 2]; }
        if (!(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(m) && isfinite(vx) && isfinite(vy) &&
              isfinite(vz)))
            atomicOr(err, ASTER_DEVERR_NONFINITE);
        pm[i] = make_double4(x, y, z, m);
        v4[i] = make_double4(vx, vy, vz, 0.0);
        float4 h, l;
        ds_split(x, h.x, l.x);
        ds_split(y, h.y, l.y);
        ds_split(z, h.z, l.z);
        h.w = __double2float_rn(m);
        l.w = 0.f;
        phi[i] = h;
        plo[i] = l;
        vf[i] = make_float4((float)vx, (float)vy, (float)vz, 0.f);
    }
}

__global__ void k_refresh_mixed(int64_t n, const double4* __restrict__ pm, const double4* __restrict__ v4,
                                float4* __restrict__ phi, float4* __restrict__ plo, float4* __restrict__ vf) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double4 p = pm[i];
        double4 v = v4[i];
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
}

// velocities and accelerations to AoS staging in one pass
__global__ void k_unpack_va(int64_t n, const double4* __restrict__ v4, const double4* __restrict__ a4,
                            double* __restrict__ dv, double* __restrict__ da) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 v = v4[i], a = a4[i];
        dv[3 * i] = v.x; dv[3 * i + 1] = v.y; dv[3 * i + 2] = v.z;
        da[3 * i] = a.x; da[3 * i + 1] = a.y; da[3 * i + 2] = a.z;
    }
}

__global__ void k_unpack3(int64_t n, const double4* __restrict__ src, double* __restrict__ dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double4 v = src[i];
        dst[3 * i] = v.x;
        dst[3 * i + 1] = v.y;
        dst[3 * i + 2] = v.z;
    }
}

// AoS double3 accelerations -> the cached double4 array (w = 0); non-finite
// values raise the error flag
__global__ void k_pack3(int64_t n, const double* __restrict__ src, double4* __restrict__ dst, int* __restrict__ err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = src[3 * i], y = src[3 * i + 1], z = src[3 * i + 2];
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) atomicOr(err, ASTER_DEVERR_NONFINITE);
        dst[i] = make_double4(x, y, z, 0.0);
    }
}

static int grid_for(aster_ctx* c, int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    int64_t cap = (int64_t)c->sm_count * 16;
    return (int)(g < cap ? (g > 0 ? g : 1) : cap);
}

int aster_refresh_mixed(aster_ctx* c) {
    k_refresh_mixed<<<grid_for(c, c->n, 256), 256, 0, c->stream>>>(
        c->n, c->pm.as<double4>(), c->vel.as<double4>(), c->phi.as<float4>(), c->plo.as<float4>(),
        c->vf.as<float4>());
    ASTER_CUDA(cudaGetLastError());
    c->mixed_valid = true;
    return ASTER_OK;
}

// Host state -> device, enqueued on the context stream (no synchronisation);
// acc (optional) becomes the cached acceleration. The host arrays must stay
// valid until the stream has consumed them.
int aster_upload_enqueue(aster_ctx* c, int64_t n, const double* pos, const double* vel, const double* mass,
                         const double* acc) {
    const size_t n4d = (size_t)n * sizeof(double4), n4f = (size_t)n * sizeof(float4);
    ASTER_TRY(c->pm.ensure(n4d));
    ASTER_TRY(c->vel.ensure(n4d));
    ASTER_TRY(c->acc.ensure(n4d));
    ASTER_TRY(c->phi.ensure(n4f));
    ASTER_TRY(c->plo.ensure(n4f));
    ASTER_TRY(c->vf.ensure(n4f));
    const size_t v3 = (size_t)n * 3 * sizeof(double);
    ASTER_TRY(c->stage.ensure(3 * v3 + (size_t)n * sizeof(double)));
    double* sp = c->stage.as<double>();
    double* sv = sp + 3 * n;
    double* sm = sv + 3 * n;
    double* sa = sm + n;
    ASTER_CUDA(cudaMemcpyAsync(sp, pos, v3, cudaMemcpyHostToDevice, c->stream));
    if (vel) ASTER_CUDA(cudaMemcpyAsync(sv, vel, v3, cudaMemcpyHostToDevice, c->stream));
    ASTER_CUDA(cudaMemcpyAsync(sm, mass, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k_pack_state<<<grid_for(c, n, 256), 256, 0, c->stream>>>(n, sp, vel ? sv : nullptr, sm, c->pm.as<double4>(),
                                                             c->vel.as<double4>(), c->phi.as<float4>(),
                                                             c->plo.as<float4>(), c->vf.as<float4>(), c->err_dev);
    ASTER_CUDA(cudaGetLastError());
    if (acc) {
        ASTER_CUDA(cudaMemcpyAsync(sa, acc, v3, cudaMemcpyHostToDevice, c->stream));
        k_pack3<<<grid_for(c, n, 256), 256, 0, c->stream>>>(n, sa, c->acc.as<double4>(), c->err_dev);
        ASTER_CUDA(cudaGetLastError());
    } else {
        ASTER_CUDA(cudaMemsetAsync(c->acc.ptr, 0, n4d, c->stream));
    }
    c->n = n;
    c->mixed_valid = true;  // k_pack_state wrote the FP32 copies
    // trailing massless bodies (test particles) attract nothing: the
    // all-pairs source loop ends at the last massive body (scanned from the end)
    int64_t last = n - 1;
    while (last > 0 && mass[last] == 0.0) --last;
    c->n_src = last + 1;
    c->acc_valid = acc != nullptr;
    c->tree.built = false;
    return ASTER_OK;
}

// Positions, velocities and accelerations into pm.xyz, vel, acc (pm.w is set
// by k_set_mass once the masses have arrived).
__global__ void k_pack_pva(int64_t n, const double* __restrict__ pos, const double* __restrict__ vel,
                           const double* __restrict__ acc, double4* __restrict__ pm, double4* __restrict__ v4,
                           double4* __restrict__ a4, int* err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        const double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
        const double ax = acc[3 * i], ay = acc[3 * i + 1], az = acc[3 * i + 2];
        if (!(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(vx) && isfinite(vy) && isfinite(vz) &&
              isfinite(ax) && isfinite(ay) && isfinite(az)))
            atomicOr(err, ASTER_DEVERR_NONFINITE);
        pm[i] = make_double4(x, y, z, 0.0);
        v4[i] = make_double4(vx, vy, vz, 0.0);
        a4[i] = make_double4(ax, ay, az, 0.0);
    }
}

// k_pack_pva followed by the first KDK step's opening kick and drift
// (v += a dt/2, x += v dt, the same operations in the same order as the
// kick-drift kernel) and the drifted bodies' bounding box: one pass over the
// staged state instead of two.
__global__ void k_pack_kick_drift(int64_t n, const double* __restrict__ pos, const double* __restrict__ vel,
                                  const double* __restrict__ acc, double half_dt, double dt,
                                  double4* __restrict__ pm, double4* __restrict__ v4, double4* __restrict__ a4,
                                  int* err, unsigned long long* __restrict__ box_bits) {
    double bmax = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double4 p = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 0.0);
        double4 v = make_double4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], 0.0);
        const double4 a = make_double4(acc[3 * i], acc[3 * i + 1], acc[3 * i + 2], 0.0);
        if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z) &&
              isfinite(a.x) && isfinite(a.y) && isfinite(a.z)))
            atomicOr(err, ASTER_DEVERR_NONFINITE);
        a4[i] = a;
        v.x += a.x * half_dt; v.y += a.y * half_dt; v.z += a.z * half_dt;
        p.x += v.x * dt; p.y += v.y * dt; p.z += v.z * dt;
        pm[i] = p;
        v4[i] = v;
        bmax = fmax(bmax, fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z))));
    }
    for (int o = 16; o > 0; o >>= 1) bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = bmax;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_xor_sync(0xffffffffu, w, o));
        // non-negative doubles order like their bit patterns
        if (threadIdx.x == 0) atomicMax(box_bits, (unsigned long long)__double_as_longlong(w));
    }
}

__global__ void k_set_mass(int64_t n, const double* __restrict__ mass, double4* __restrict__ pm, int* err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double m = mass[i];
        if (!isfinite(m)) atomicOr(err, ASTER_DEVERR_NONFINITE);
        pm[i].w = m;
    }
}

// Host state -> device for a step on the tree solver, with the masses' copy
// off the critical path: positions, velocities and accelerations go first,
// back to back on the context stream; the masses follow on the copy stream
// and arrive while the kick-drift, bounding box, Morton codes and sort run
// (none of which reads a mass). aster_apply_pending_mass, called by the tree
// build before its first mass read, waits for them. The FP32 copies are not
// written (the tree path does not read them). Requires c->copy_stream.
int aster_upload_enqueue_overlapped(aster_ctx* c, int64_t n, const double* pos, const double* vel, const double* mass,
                                    const double* acc, const aster_params* kick_drift) {
    const size_t n4d = (size_t)n * sizeof(double4), n4f = (size_t)n * sizeof(float4);
    ASTER_TRY(c->pm.ensure(n4d));
    ASTER_TRY(c->vel.ensure(n4d));
    ASTER_TRY(c->acc.ensure(n4d));
    ASTER_TRY(c->phi.ensure(n4f));
    ASTER_TRY(c->plo.ensure(n4f));
    ASTER_TRY(c->vf.ensure(n4f));
    const size_t v3 = (size_t)n * 3 * sizeof(double);
    ASTER_TRY(c->stage.ensure(3 * v3 + (size_t)n * sizeof(double)));
    double* sp = c->stage.as<double>();
    double* sv = sp + 3 * n;
    double* sm = sv + 3 * n;
    double* sa = sm + n;
    ASTER_CUDA(cudaMemcpyAsync(sp, pos, v3, cudaMemcpyHostToDevice, c->stream));
    ASTER_CUDA(cudaMemcpyAsync(sv, vel, v3, cudaMemcpyHostToDevice, c->stream));
    ASTER_CUDA(cudaMemcpyAsync(sa, acc, v3, cudaMemcpyHostToDevice, c->stream));
    ASTER_CUDA(cudaEventRecord(c->ev[3], c->stream));
    ASTER_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev[3], 0));
    ASTER_CUDA(cudaMemcpyAsync(sm, mass, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->copy_stream));
    ASTER_CUDA(cudaEventRecord(c->ev[4], c->copy_stream));
    if (kick_drift) {
        ASTER_TRY(c->red.ensure(4096));
        ASTER_CUDA(cudaMemsetAsync(red_box(c), 0, sizeof(unsigned long long), c->stream));
        k_pack_kick_drift<<<grid_for(c, n, 256), 256, 0, c->stream>>>(
            n, sp, sv, sa, 0.5 * kick_drift->dt, kick_drift->dt, c->pm.as<double4>(), c->vel.as<double4>(),
            c->acc.as<double4>(), c->err_dev, red_box(c));
    } else {
        k_pack_pva<<<grid_for(c, n, 256), 256, 0, c->stream>>>(n, sp, sv, sa, c->pm.as<double4>(),
                                                               c->vel.as<double4>(), c->acc.as<double4>(), c->err_dev);
    }
    ASTER_CUDA(cudaGetLastError());
    c->mass_pending = sm;
    c->n = n;
    c->mixed_valid = false;
    int64_t last = n - 1;
    while (last > 0 && mass[last] == 0.0) --last;
    c->n_src = last + 1;
    c->acc_valid = true;
    c->tree.built = false;
    return ASTER_OK;
}

int aster_apply_pending_mass(aster_ctx* c) {
    if (!c->mass_pending) return ASTER_OK;
    ASTER_CUDA(cudaStreamWaitEvent(c->stream, c->ev[4], 0));
    k_set_mass<<<grid_for(c, c->n, 256), 256, 0, c->stream>>>(c->n, c->mass_pending, c->pm.as<double4>(), c->err_dev);
    ASTER_CUDA(cudaGetLastError());
    c->mass_pending = nullptr;
    return ASTER_OK;
}

static int state_upload(aster_ctx* c, int64_t n, const double* pos, const double* vel, const double* mass,
                        const double* acc) {
    if (!c || !pos || !mass || n <= 0 || n > (int64_t)1 << 30) return ASTER_ERR_INVALID_ARG;
    ASTER_TRY(aster_begin(c));
    int st = aster_upload_enqueue(c, n, pos, vel, mass, acc);
    if (st == ASTER_OK) st = aster_finish(c);
    if (st != ASTER_OK) {
        c->n = 0;
        c->acc_valid = false;
    }
    return st;
}

// One of the state arrays (0 positions, 1 velocities, 2 accelerations) ->
// host AoS double3 through the staging area, on `stream` (no synchronisation).
int aster_download_enqueue(aster_ctx* c, int which, double* host, cudaStream_t stream) {
    const int64_t n = c->n;
    const size_t v3 = (size_t)n * 3 * sizeof(double);
    const DevBuf* srcs[3] = {&c->pm, &c->vel, &c->acc};
    double* st = c->stage.as<double>() + 3 * n * which;
    k_unpack3<<<grid_for(c, n, 256), 256, 0, stream>>>(n, srcs[which]->as<double4>(), st);
    ASTER_CUDA(cudaGetLastError());
    ASTER_CUDA(cudaMemcpyAsync(host, st, v3, cudaMemcpyDeviceToHost, stream));
    return ASTER_OK;
}

// Velocities and accelerations -> host: one unpack kernel, then the two copies
// back to back (no kernel between the transfers).
int aster_download_va_enqueue(aster_ctx* c, double* vel, double* acc, cudaStream_t stream) {
    const int64_t n = c->n;
    const size_t v3 = (size_t)n * 3 * sizeof(double);
    double* sv = c->stage.as<double>() + 3 * n;
    double* sa = sv + 3 * n;
    k_unpack_va<<<grid_for(c, n, 256), 256, 0, stream>>>(n, c->vel.as<double4>(), c->acc.as<double4>(), sv, sa);
    ASTER_CUDA(cudaGetLastError());
    ASTER_CUDA(cudaMemcpyAsync(vel, sv, v3, cudaMemcpyDeviceToHost, stream));
    ASTER_CUDA(cudaMemcpyAsync(acc, sa, v3, cudaMemcpyDeviceToHost, stream));
    return ASTER_OK;
}

extern "C" int aster_state_upload(aster_ctx* c, int64_t n, const double* pos, const double* vel,
                                  const double* mass) {
    return state_upload(c, n, pos, vel, mass, nullptr);
}

extern "C" int aster_state_upload_acc(aster_ctx* c, int64_t n, const double* pos, const double* vel,
                                      const double* mass, const double* acc) {
    if (!acc) return ASTER_ERR_INVALID_ARG;
    return state_upload(c, n, pos, vel, mass, acc);
}

extern "C" int aster_state_download(aster_ctx* c, double* pos, double* vel, double* acc) {
    if (!c) return ASTER_ERR_INVALID_ARG;
    if (c->n <= 0) return ASTER_ERR_NO_STATE;
    ASTER_CUDA(cudaSetDevice(c->device));
    const int64_t n = c->n;
    const size_t v3 = (size_t)n * 3 * sizeof(double);
    ASTER_TRY(c->stage.ensure(3 * v3));
    double* st = c->stage.as<double>();
    const DevBuf* srcs[3] = {&c->pm, &c->vel, &c->acc};
    double* dsts[3] = {pos, vel, acc};
    for (int k = 0; k < 3; ++k) {
        if (!dsts[k]) continue;
        k_unpack3<<<grid_for(c, n, 256), 256, 0, c->stream>>>(n, srcs[k]->as<double4>(), st + 3 * n * k);
        ASTER_CUDA(cudaGetLastError());
        ASTER_CUDA(cudaMemcpyAsync(dsts[k], st + 3 * n * k, v3, cudaMemcpyDeviceToHost, c->stream));
    }
    ASTER_CUDA(cudaStreamSynchronize(c->stream));
    return ASTER_OK;
}

extern "C" int aster_state_size(aster_ctx* c, int64_t* n) {
    if (!c || !n) return ASTER_ERR_INVALID_ARG;
    *n = c->n;
    return ASTER_OK;
}

int aster_copy_acc_out(aster_ctx* c, double* acc_out) {
    if (!acc_out) return ASTER_OK;
    return aster_state_download(c, nullptr, nullptr, acc_out);
}

extern "C" int aster_get_stats(aster_ctx* c, aster_stats* out) {
    if (!c || !out) return ASTER_ERR_INVALID_ARG;
    *out = c->stats;
    return ASTER_OK;
}
