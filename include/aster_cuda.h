/*
 * aster_cuda.h -- C ABI of the B200 (sm_100a) force-evaluation and integration
 * hot path for Aster. Plain C types only: no CUDA, torch or C++ types cross
 * this boundary. Every function returns an int status (ASTER_OK or an
 * ASTER_ERR_* code) and never exits the process.
 *
 * Pointer convention: every pointer is HOST memory unless its name ends in
 * `_dev`. Vectors are array-of-structs FP64 triples (x,y,z per body), which is
 * the reference's BodyArray layout (include/Aster/physics/body.h:9-24,
 * std::vector<vec3> of doubles, include/Aster/physics/vectors.h:44-75).
 *
 * Reference interfaces replaced (paths within the reference project):
 *   Solver::compute_forces          include/Aster/simulations/sim_obj.h:34-61
 *   Parallelized::compute_forces    src/utils/builder_endpoint.cpp:729-757
 *   SimpleGPU::compute_forces       src/solvers/SimpleGPU.cpp:17-71
 *   Barnes_Hut::make_tree/compute_forces  src/solvers/barnes_hut.cpp:309-418
 *   BH_hyper::compute_forces        src/solvers/full_GPU.cpp:519-527
 *   update_leapfrog(_gpu_3d)        src/physics/tool_chain_impl.cpp:169-185,
 *                                   src/utils/updater.cpp:53-87
 *   Simulation::load_gpu_buffers / read_bodies_gpu
 *                                   src/utils/builder_endpoint.cpp:102-119,424-434
 *   Graphs::get_total_energy        src/utils/collectors.cpp:19-53
 */
#ifndef ASTER_CUDA_H
#define ASTER_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define ASTER_OK 0
#define ASTER_ERR_INVALID_ARG 1    /* null pointer, bad enum, n out of range   */
#define ASTER_ERR_CUDA 2           /* a CUDA runtime call failed               */
#define ASTER_ERR_OOM 3            /* device allocation failed                 */
#define ASTER_ERR_NO_STATE 4       /* no bodies uploaded yet                   */
#define ASTER_ERR_STACK 5          /* tree-walk stack overflow (walk stopped)  */
#define ASTER_ERR_TREE 6           /* bottom-up climb exceeded its level cap   */
#define ASTER_ERR_NONFINITE 7      /* NaN/Inf found in inputs or results       */
#define ASTER_ERR_CANCELLED 8      /* persistent kernel stopped by cancel flag */
#define ASTER_ERR_UNSUPPORTED 9    /* option combination not implemented       */
#define ASTER_ERR_TOO_LARGE 10     /* size beyond a fixed capacity             */
#define ASTER_ERR_KEPLER 11        /* Kepler drift: no convergence, or a body at
                                      the central mass's position             */

/* ---- force law bits: the reference PN_expansion_type bitmask
 *      (include/Aster/simulations/basic.h:39-53) ------------------------- */
#define ASTER_NEWTON 0x0001
#define ASTER_PN1 0x0010  /* get_pn1, c^-2 (src/physics/tool_chain_impl.cpp:110-118)  */
#define ASTER_PN2 0x0100  /* get_pn2, c^-4 (tool_chain_impl.cpp:79-107); all-pairs and ensemble */
#define ASTER_PN25 0x1000 /* get_pn25, c^-5 (tool_chain_impl.cpp:65-77); all-pairs and ensemble */
/* Not a reference bit: with ASTER_PN1, the 1PN term is the N-body
 * Einstein-Infeld-Hoffmann acceleration (the pairwise get_pn1 terms plus the
 * three-body couplings it leaves out). Ensemble entry points only, without
 * ASTER_PN2/ASTER_PN25; every other entry point returns ASTER_ERR_UNSUPPORTED. */
#define ASTER_EIH 0x10000

/* ---- enums ------------------------------------------------------------- */
#define ASTER_FP64 0   /* plain FP64 pair arithmetic                          */
#define ASTER_MIXED 1  /* FP32 pair arithmetic on double-single relative
                          positions, compensated accumulation, FP64 results   */

#define ASTER_SOLVER_ALLPAIRS 0 /* replaces Parallelized / SimpleGPU          */
#define ASTER_SOLVER_LBVH 1     /* replaces Barnes_Hut / BH_hyper             */

typedef struct aster_ctx aster_ctx; /* opaque: device state + scratch        */

/* Physical and algorithmic parameters. The reference reads these from the
 * Simulation (sim_obj.h:165-180, sim_meta.h:8-60); here they are explicit. */
typedef struct aster_params {
    double G;           /* gravitational constant (Simulation::get_G)          */
    double c;           /* speed of light, used by PN terms (get_c)            */
    double eps2;        /* softening added to r^2 (Simulation::softening)      */
    double theta;       /* opening angle (Simulation::theta)                   */
    double dt;          /* time step (get_dt)                                  */
    int32_t force_law;  /* ASTER_NEWTON | ASTER_PN1 [| ASTER_PN2 | ASTER_PN25]   */
    int32_t morton_bits;/* 30 (reference) or 63                                */
    int32_t compat_mode;/* 1: OpenCL BH_hyper tree semantics (descending order,
                           body-index tie-break, 1024->0 Morton wrap)         */
    int32_t reserved;   /* must be 0                                           */
} aster_params;

/* Tree arrays in the reference's layout (barnes_hut.cpp:338-396): leaves
 * 0..n-1 in sorted order, internal nodes n..2n-2, root = n, -1 = no child.
 * Every pointer is host memory of the stated length, or NULL to skip. */
typedef struct aster_tree_view {
    uint64_t* codes;        /* [n]  Morton code per body, input order        */
    uint64_t* sorted_codes; /* [n]  codes in sorted order                    */
    int32_t* perm;          /* [n]  body index of each sorted leaf           */
    int32_t* left;          /* [2n-1]                                        */
    int32_t* right;         /* [2n-1]                                        */
    int32_t* parent;        /* [2n-1] (parent[root] = -1)                    */
    int32_t* range_lo;      /* [2n-1] first sorted leaf under the node       */
    int32_t* range_hi;      /* [2n-1] last sorted leaf under the node        */
    double* node_mass;      /* [2n-1] FP64 (NodesArray::masses)              */
    double* node_com;       /* [(2n-1)*3] FP64 (NodesArray::centers_of_mass) */
    float* node_bmin;       /* [(2n-1)*3] FP32 AABB, rounded outwards        */
    float* node_bmax;       /* [(2n-1)*3]                                    */
    float* node_rcrit2;     /* [2n-1] squared opening radius (leaves 0)      */
    double box;             /* out: Morton cube half-width used              */
} aster_tree_view;

/* Timing and work counters of the last call that filled them. */
typedef struct aster_stats {
    double ms_total;          /* device time of the call (CUDA events)        */
    double ms_force;          /* of which the force kernel                    */
    double ms_build;          /* of which the LBVH build                      */
    double interactions;      /* pair interactions evaluated                  */
    int32_t max_stack;        /* tree-walk stack high-water mark              */
    int32_t kernels;          /* kernel launches issued                       */
} aster_stats;

const char* aster_strerror(int status);
int aster_version(void);

/* Create a context on CUDA device `device`. `stream` is a cudaStream_t cast
 * to void*, or NULL for a stream owned by the context. */
int aster_ctx_create(aster_ctx** out, int device, void* stream);
int aster_ctx_destroy(aster_ctx* ctx);

/* Host -> device copy of the body state (Simulation::load_gpu_buffers,
 * builder_endpoint.cpp:102-119). vel may be NULL (zero velocities).
 * Invalidates the cached acceleration. */
int aster_state_upload(aster_ctx* ctx, int64_t n, const double* pos,
                       const double* vel, const double* mass);
/* aster_state_upload plus the bodies' current accelerations (AoS double3, the
 * reference's BodyArray::accs): they become the cached acceleration, so the
 * next KDK step starts with its kick instead of a force evaluation, as a
 * device-resident run would. acc must be the acceleration of these positions
 * under the next call's parameters (what aster_state_download returned after
 * a KDK call, or the reference update_leapfrog's a(x_{n+1})). */
int aster_state_upload_acc(aster_ctx* ctx, int64_t n, const double* pos,
                           const double* vel, const double* mass, const double* acc);
/* Device -> host copy (read_bodies_gpu, builder_endpoint.cpp:424-434); any
 * pointer may be NULL. acc is the cached acceleration of the current state. */
int aster_state_download(aster_ctx* ctx, double* pos, double* vel, double* acc);
int aster_state_size(aster_ctx* ctx, int64_t* n);

/* One all-pairs force evaluation of the current state (skips j == i), the
 * Parallelized / SimpleGPU replacement. Accelerations are cached on the device
 * and copied to acc_out (host, n*3) when it is not NULL. */
int aster_allpairs(aster_ctx* ctx, const aster_params* p, int precision, double* acc_out);
/* Accelerations of every body from the sources [src_lo, src_hi) only
 * (src_hi < 0: up to n): Parallelized::compute_forces over a Solver::set_bounds
 * range (builder_endpoint.cpp:64-69, 729-757), e.g. set_bounds(1, -1) in
 * update_WH_planetary (updater.cpp:100). acc_out: host, n*3, or NULL. The
 * cached acceleration is not the full one afterwards (the next KDK step
 * evaluates it afresh). */
int aster_allpairs_range(aster_ctx* ctx, const aster_params* p, int precision, int64_t src_lo, int64_t src_hi,
                         double* acc_out);

/* All-pairs accelerations for an explicit target list against every body:
 * targets[nt] body indices, acc_out[nt*3] host. FP64 or mixed. Used for the
 * sampled accuracy check of the tree code at large n. */
int aster_allpairs_targets(aster_ctx* ctx, const aster_params* p, int precision,
                           int64_t nt, const int32_t* targets, double* acc_out);

/* Build the LBVH of the current state (Morton -> stable radix sort ->
 * Karras tree -> bottom-up moments/bounds). view may be NULL; its non-NULL
 * arrays are filled. */
int aster_lbvh_build(aster_ctx* ctx, const aster_params* p, aster_tree_view* view);

/* Build + warp-group traversal (Barnes_Hut / BH_hyper compute_forces
 * replacement). A group is a subtree of at most 64 leaves whose parent holds
 * more; one warp walks the tree once per group. precision: ASTER_MIXED (FP32
 * interactions) or ASTER_FP64 (same tree, same interaction lists, FP64
 * arithmetic). acc_out may be NULL. list_counts (host, n, input order)
 * receives the interaction-list length of each body's group when not NULL. */
int aster_lbvh_forces(aster_ctx* ctx, const aster_params* p, int precision,
                      double* acc_out, int32_t* list_counts);

/* nsteps kick-drift-kick leapfrog steps of the resident state with one force
 * evaluation per step (the acceleration is cached across steps; the reference
 * update_leapfrog evaluates twice per step). solver: ASTER_SOLVER_*. With
 * the tree solver, the steps between the first and the last run as launches
 * of one CUDA graph that the context keeps until it is destroyed: a later call
 * with the same parameters, body count and device buffers launches it again
 * instead of capturing a new one. */
int aster_kdk_steps(aster_ctx* ctx, const aster_params* p, int solver, int precision,
                    int nsteps);

/* Host-resident loop in one call: uploads (pos, vel, mass, acc), takes
 * nsteps >= 1 KDK steps and writes pos, vel, acc back (n bodies, AoS double3,
 * acc = the accelerations of pos on input and output, as
 * aster_state_upload_acc expects). The copy of the final positions to the host
 * overlaps the last force evaluation. Use pinned host memory for the copies
 * to run asynchronously. The resident state is the stepped state afterwards. */
int aster_kdk_steps_host(aster_ctx* ctx, const aster_params* p, int solver, int precision,
                         int nsteps, int64_t n, double* pos, double* vel, double* acc,
                         const double* mass);

/* nsteps of the symplectic SABA_order integrator (order 1..10) on the
 * resident state. Replaces update_SABA1..10 (src/integrators/SABA.cpp:14-553)
 * and the OpenCL SABA updater (src/utils/tc_impl_cl.cpp:269-299). Order n >= 2:
 * drift c_1, then n times (forces, kick d_k, drift c_{k+1}) with the Laskar-
 * Robutel coefficients (Gauss-Legendre nodes and weights on [0,1]); order 1
 * is the reference's SABA1 = update_euler (forces, v += a dt, x += v dt).
 * n force evaluations per step; the cached acceleration is invalidated. */
int aster_saba_steps(aster_ctx* ctx, const aster_params* p, int solver, int precision,
                     int order, int nsteps);

/* nsteps of the Wisdom-Holman planetary integrator: body 0 is the central mass
 * (positive), every other body moves on a Kepler orbit about it (universal
 * variables, on the device) perturbed by the others' Newtonian attraction (the
 * all-pairs kernel at `precision`, softened by eps2). Democratic heliocentric
 * splitting, one interaction evaluation per step. Replaces update_WH_planetary
 * (src/physics/tool_chain_impl.cpp:186-290) and its OpenCL form
 * (include/Aster/kernels/WH_planetary.cl.h), whose kick re-applies the
 * central attraction. Newtonian force law only. ASTER_ERR_KEPLER when a Kepler
 * drift does not converge or a body sits on the central mass (that body is
 * then left undrifted). The cached acceleration is invalidated. */
int aster_wh_steps(aster_ctx* ctx, const aster_params* p, int precision, int nsteps);

/* ---- device-resident stepping with recorded time series ---------------
 * Replaces Simulation::step/integrate with its Graph collectors
 * (src/utils/builder_endpoint.cpp:274-352, src/utils/graph_collection.cpp,
 * src/utils/collectors.cpp): the reference reads the bodies back every step
 * and evaluates the collectors on the host; here the updater advances the
 * resident state `rate` steps at a time, collector kernels write one row per
 * sample into a device table, and the table is copied back once. */
#define ASTER_UPDATER_KDK 0   /* aster_kdk_steps                            */
#define ASTER_UPDATER_SABA 1  /* aster_saba_steps (order)                   */
#define ASTER_UPDATER_WH 2    /* aster_wh_steps (body 0 central)            */

#define ASTER_COLLECT_ENERGY 0x1        /* hamiltonian_collector: total energy */
#define ASTER_COLLECT_ENERGY_ERROR 0x2  /* error_collector: |E - E0| / |E0|, E0 at the start */
#define ASTER_COLLECT_MOMENTUM 0x4      /* total momentum (3 columns)          */
#define ASTER_COLLECT_CENTER 0x8        /* centre of mass (3 columns)          */
#define ASTER_COLLECT_DISTANCE 0x10     /* distance_collector: |x_cm - x_b + 0.1| per body (n columns) */

typedef struct aster_record_config {
    int32_t updater;    /* ASTER_UPDATER_*                                     */
    int32_t order;      /* SABA order 1..10 (ASTER_UPDATER_SABA)              */
    int32_t solver;     /* ASTER_SOLVER_* (KDK, SABA; WH uses all-pairs)       */
    int32_t precision;  /* ASTER_FP64 or ASTER_MIXED                           */
    int32_t rate;       /* a sample after every `rate` steps (>= 1)           */
    int32_t collect;    /* ASTER_COLLECT_* bits                                */
    int32_t ref_form;   /* energy with the reference formula (1) or Plummer (0) */
    int32_t reserved;   /* 0                                                   */
} aster_record_config;

/* Columns of one recorded row: time + the collected quantities, in the order
 * of the bits above (the per-body distances last). */
int64_t aster_record_columns(const aster_record_config* cfg, int64_t n);

/* nsteps with cfg->updater, sampling at steps 0, rate, 2 rate, ... (nsteps /
 * rate + 1 rows; any steps after the last sample are still taken). rows_out
 * (host): rows x aster_record_columns doubles, row-major, each row
 * [step, columns...] -- the rows of the reference's Graph CSV files. */
int aster_record(aster_ctx* ctx, const aster_params* p, const aster_record_config* cfg, int64_t nsteps,
                 double* rows_out);

/* FP64 diagnostics of the current state: total energy with the Plummer
 * potential -G m_i m_j / sqrt(r^2 + eps2) (consistent with the force), total
 * momentum p[3]. ref_form = 1 uses the reference formula
 * -G m_i m_j / (r + eps2) of collectors.cpp:43 instead. */
int aster_energy(aster_ctx* ctx, const aster_params* p, int ref_form, double* energy,
                 double* momentum3);

/* ---- batched ensembles of few-body systems ------------------------------
 * Thousands of independent systems of 1..64 bodies integrated by one
 * persistent kernel (one warp per system, systems taken largest first from a
 * work counter), launched through a captured CUDA graph. The pair law is the
 * reference's (compute_gravitational / get_pn1, tool_chain_impl.cpp:110-137,
 * Newton + optional pairwise 1PN, 2PN, 2.5PN), or with ASTER_EIH the N-body
 * Einstein-Infeld-Hoffmann 1PN acceleration; the integrators are compositions of
 * drift-kick-drift leapfrog steps: the reference's leapfrog
 * (tool_chain_impl.cpp:169-185, same map) and Yoshida's (1990) fourth-order
 * triple jump, which the reference lacks. The reference has no batched
 * solver; per-system Simulations would also share Parallelized's cached
 * pointer (builder_endpoint.cpp:731). */
#define ASTER_INTEGRATOR_LEAPFROG 0
#define ASTER_INTEGRATOR_YOSHIDA4 1
#define ASTER_ENSEMBLE_MAX_BODIES 64

typedef struct aster_ensemble_config {
    int32_t warps_per_block; /* 1..16 (0: 4)                                  */
    int32_t unroll;          /* inner-loop unroll 1, 2 or 4 (0: 2)            */
    int32_t check_every;     /* steps between cancel-flag reads (0: 256)      */
    int32_t use_graph;       /* 1: capture the launch in a CUDA graph         */
    int32_t schedule;        /* order warps take systems in: 0 largest first
                                (longest-processing-time), 1 upload order     */
} aster_ensemble_config;

/* offsets[nsys+1]: system s owns bodies offsets[s] .. offsets[s+1]-1 of the
 * AoS FP64 arrays (1 <= size <= 64). vel may be NULL. */
int aster_ensemble_upload(aster_ctx* ctx, int32_t nsys, const int64_t* offsets, const double* pos,
                          const double* vel, const double* mass);
int aster_ensemble_download(aster_ctx* ctx, double* pos, double* vel);
/* nsteps steps of every system in one launch. precision: ASTER_MIXED (FP64
 * state, FP32 pair terms on double-single separations) or ASTER_FP64.
 * cfg may be NULL (defaults). Returns ASTER_ERR_CANCELLED if
 * aster_ensemble_cancel was called meanwhile (systems stop at a step
 * boundary that is a multiple of check_every). */
int aster_ensemble_run(aster_ctx* ctx, const aster_params* p, int integrator, int precision, int64_t nsteps,
                       const aster_ensemble_config* cfg);
/* FP64 energy per system (energy[nsys]): Newtonian with the softened
 * potential, plus, when the force law has the PN1 bit, the 1PN energy of the
 * EIH Lagrangian: with ASTER_EIH its full N-body form (the energy the EIH
 * equations conserve to order c^-4), otherwise the sum of its two-body
 * terms over pairs. */
int aster_ensemble_energy(aster_ctx* ctx, const aster_params* p, double* energy);
/* Thread-safe request to stop a running aster_ensemble_run. */
int aster_ensemble_cancel(aster_ctx* ctx);

/* ---- adjoint of the kick-drift-kick leapfrog ----------------------------
 * Loss L = (1/n) sum_i |x_T,i - target_i|^2 after nsteps KDK steps (the
 * aster_kdk_steps map, Newtonian all-pairs forces) from the uploaded state,
 * and its gradients dL/dx0, dL/dv0 (host, n*3) and dL/dm (host, n) by a
 * hand-written reverse sweep: the forward pass stores (x, v, a) every
 * checkpoint_every steps; the reverse pass recomputes each segment from its
 * checkpoint and runs the adjoint recurrences
 *   lv' = lv + dt lx;  w = c h lv';  lx += J(x_n)^T w;  lm += (dA/dm)^T w
 * (h = dt/2, c = 2 except at n = 0) with one O(N^2) tidal-tensor/vector kernel
 * per step. precision ASTER_MIXED: FP32 pair arithmetic (forces and adjoint),
 * FP64 state and adjoint variables; ASTER_FP64: FP64 throughout. The uploaded
 * state is unchanged on return. The reference has no adjoint. Any output
 * pointer may be NULL. */
int aster_adjoint_leapfrog(aster_ctx* ctx, const aster_params* p, int precision, int64_t nsteps,
                           int32_t checkpoint_every, const double* target, double* loss, double* grad_x0,
                           double* grad_v0, double* grad_m);

/* Allocation-free energy. No counterpart in the reference.
 *
 * For callers that cannot allocate device memory: codes that reserve all of
 * the GPU's memory up front in their own pool (a cudaMalloc would fail or
 * break their accounting), and time-stepping loops that must not allocate in
 * the middle of a run because an allocation or free can stall the whole
 * device. It computes what aster_energy computes, but takes device arrays from
 * the caller and needs no context:
 *   pm_dev   n records of 4 doubles (x, y, z, m), 32-byte aligned
 *   vel_dev  n records of 4 doubles (vx, vy, vz, unused), 32-byte aligned
 *   out_dev  4 doubles: total energy, then the momentum (px, py, pz)
 * The per-block partial sums live in a fixed array inside the library (2.5 MiB
 * on every GPU that loads it, held until the process exits), so n is limited
 * to ASTER_ENERGY_NOALLOC_MAX_N; larger n returns ASTER_ERR_TOO_LARGE. The
 * work is queued on `stream` (a cudaStream_t, NULL for the default stream) and
 * the call returns without waiting; synchronise before reading out_dev.
 * The first call on a device looks up that device's address of the array, so
 * make that first call before any stream capture. The address is kept for the
 * life of the process: calling cudaDeviceReset after the first call on that
 * device is not supported (the module is reloaded elsewhere and the kept
 * address goes stale). Every block adds up 256 bodies against all sources in
 * one launch, so below about 40,000 bodies the GPU is only partly filled and
 * this call is several times slower than aster_energy, which also splits the
 * sources over blocks. All calls share the one
 * array: calls that overlap on the GPU (on different streams) race and give
 * wrong results. Each call fully rewrites the partials it reads, so nothing
 * needs clearing between calls. */
#define ASTER_ENERGY_NOALLOC_MAX_N (65536LL * 256)
int aster_energy_noalloc(int64_t n, const double* pm_dev, const double* vel_dev, const aster_params* p,
                         int ref_form, double* out_dev, void* stream);

/* Counters of the last force/step call on this context. */
int aster_get_stats(aster_ctx* ctx, aster_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* ASTER_CUDA_H */
