// Implementation of the Aster Solver/Updater binding over the C ABI.
#include "aster_cuda_solvers.h"

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>
#include <string>

namespace Aster {

void CudaSolverBase::check(int status, const char* where) {
    if (status == ASTER_OK) return;
    // the reference reports GPU errors through critical_if (logging.cpp:32-47)
    critical_if(true, std::string(where) + ": " + aster_strerror(status));
}

CudaSolverBase::~CudaSolverBase() {
    if (ctx_) aster_ctx_destroy(ctx_);
}

void CudaSolverBase::ensure_context() {
    if (!ctx_) check(aster_ctx_create(&ctx_, device_, nullptr), "aster_ctx_create");
}

aster_params CudaSolverBase::params() const {
    aster_params p{};
    p.G = sim_->get_G();
    p.c = sim_->get_c();
    p.eps2 = sim_->softening;
    p.theta = sim_->theta;
    p.dt = sim_->get_dt();
    p.force_law = self_->force_law.type & (ASTER_NEWTON | ASTER_PN1 | ASTER_PN2 | ASTER_PN25);
    p.morton_bits = 30;
    p.compat_mode = 0;
    p.reserved = 0;
    return p;
}

void CudaSolverBase::upload() {
    ensure_context();
    auto& b = sim_->bodies;
    const int64_t n = (int64_t)b.positions.size();
    // vec3 is three packed doubles (include/Aster/physics/vectors.h:44-75)
    check(aster_state_upload(ctx_, n, &b.positions[0].x, b.velocities.empty() ? nullptr : &b.velocities[0].x,
                             b.masses.data()),
          "aster_state_upload");
}

CudaAllPairs::CudaAllPairs(Simulation* s, int precision, int device)
    : CudaSolverBase(s, this, precision, device) {
    this->_s = s;
    this->type = SIMPLE_GPU;
}

void CudaAllPairs::compute_forces() {
    auto& b = _s->bodies;
    if (b.positions.empty()) return;
    // set_bounds restricts the sources, as in Parallelized::compute_forces
    // (builder_endpoint.cpp:729-757): every body gets the pull of [lower, upper)
    const int lo = get_lower_bound(), hi = get_upper_bound();
    if (warn_if(hi - lo <= 0, "either upper or lower bound were set too high in the gravity solver, resulting in a negative amount of bodies to load"))
        return;
    upload();
    b.accs.resize(b.positions.size());
    const aster_params p = params();
    if (lo != 0 || hi != (int)b.positions.size())
        check(aster_allpairs_range(ctx_, &p, precision_, lo, hi, &b.accs[0].x), "aster_allpairs_range");
    else
        check(aster_allpairs(ctx_, &p, precision_, &b.accs[0].x), "aster_allpairs");
}

CudaLBVH::CudaLBVH(Simulation* s, int precision, int device) : CudaSolverBase(s, this, precision, device) {
    this->_s = s;
    this->type = GPU_BARNES_HUT;
    this->num_childs = 2;
}

void CudaLBVH::compute_forces() {
    auto& b = _s->bodies;
    if (b.positions.empty()) return;
    // Barnes_Hut::compute_forces with bounds builds its tree from misnumbered
    // bodies (make_tree stores i - lower as the body index and keeps the root
    // at N): there is no consistent meaning to reproduce, so ranges are refused
    if (get_lower_bound() != 0 || get_upper_bound() != (int)b.positions.size()) {
        critical_if(true, "CudaLBVH: set_bounds ranges are not supported; use CudaAllPairs for a source range");
        return;
    }
    upload();
    b.accs.resize(b.positions.size());
    const aster_params p = params();
    check(aster_lbvh_forces(ctx_, &p, precision_, &b.accs[0].x, nullptr), "aster_lbvh_forces");
    if (keep_tree) sync_tree();
}

void CudaLBVH::sync_tree() {
    auto& b = _s->bodies;
    const size_t n = b.positions.size();
    bounding_box = _s->get_center() * 2;  // as make_tree records it (barnes_hut.cpp:317)
    compressed_mortons_size = (long)n;
    if (n == 0) return;
    auto leaf = [&](size_t i, size_t body) {
        nodes.masses[i] = b.masses[body];
        nodes.centers_of_mass[i] = b.positions[body];
        nodes.velocities[i] = b.velocities.empty() ? vec3(0.0) : b.velocities[body];
        nodes.temps[i] = b.temps.size() > body ? b.temps[body] : 0.0;
        nodes.left_nodes[i] = nodes.right_nodes[i] = -1;
    };
    if (n == 1) {  // make_tree builds nothing for one body; its only node is the body
        nodes.resize(1);
        leaf(0, 0);
        return;
    }
    upload();
    const size_t m = 2 * n - 1;
    std::vector<int32_t> perm(n), left(m), right(m);
    std::vector<double> mass(m), com(3 * m);
    aster_tree_view v{};
    v.perm = perm.data();
    v.left = left.data();
    v.right = right.data();
    v.node_mass = mass.data();
    v.node_com = com.data();
    const aster_params p = params();
    check(aster_lbvh_build(ctx_, &p, &v), "aster_lbvh_build");
    nodes.resize(m);
    for (size_t i = 0; i < n; ++i) leaf(i, (size_t)perm[i]);
    for (size_t i = 0; i < m; ++i) {
        nodes.left_nodes[i] = left[i];
        nodes.right_nodes[i] = right[i];
        nodes.masses[i] = mass[i];
        nodes.centers_of_mass[i] = vec3(com[3 * i], com[3 * i + 1], com[3 * i + 2]);
    }
    // velocities and temps of the internal nodes as NodesArray::unite forms
    // them (barnes_hut.cpp:137-152), children first: post-order from the root
    std::vector<std::pair<int32_t, bool>> st{{(int32_t)n, false}};
    while (!st.empty()) {
        auto [k, expanded] = st.back();
        st.pop_back();
        if (k < (int32_t)n) continue;
        const int32_t L = left[k], R = right[k];
        if (!expanded) {
            st.push_back({k, true});
            st.push_back({R, false});
            st.push_back({L, false});
            continue;
        }
        const double M = mass[k];
        if (M > 0.0)
            nodes.velocities[k] = (nodes.velocities[R] * mass[R] + nodes.velocities[L] * mass[L]) / M;
        else  // no mass below: the children's mean, like the centre the device gives such a node
            nodes.velocities[k] = (nodes.velocities[R] + nodes.velocities[L]) * 0.5;
        nodes.temps[k] = std::max(nodes.temps[R], nodes.temps[L]);
    }
}

// The base Updater is constructed as a leapfrog (a valid entry of
// integrator_mapper, updater.cpp:20-25); update_bodies() replaces it.
CudaKDK::CudaKDK(Simulation* s, CudaSolverBase* solver) : Updater(s, 0, LEAPFROG), solver_(solver) {}

void CudaKDK::update_bodies() {
    auto& b = _s->bodies;
    if (b.positions.empty()) return;
    if (!uploaded_) {
        solver_->upload();
        uploaded_ = true;
    }
    const aster_params p = solver_->params();
    aster_ctx* ctx = solver_->context();
    int st = aster_kdk_steps(ctx, &p, solver_->solver_kind(), solver_->precision(), 1);
    if (st == ASTER_OK) {
        b.accs.resize(b.positions.size());
        st = aster_state_download(ctx, &b.positions[0].x, &b.velocities[0].x, &b.accs[0].x);
    }
    if (st != ASTER_OK) critical_if(true, std::string("CudaKDK: ") + aster_strerror(st));
}

CudaSABA::CudaSABA(Simulation* s, CudaSolverBase* solver, int order)
    : Updater(s, order - 1, SABA), solver_(solver), saba_order_(order) {}

void CudaSABA::update_bodies() {
    auto& b = _s->bodies;
    if (b.positions.empty()) return;
    if (!uploaded_) {
        solver_->upload();
        uploaded_ = true;
    }
    const aster_params p = solver_->params();
    aster_ctx* ctx = solver_->context();
    int st = aster_saba_steps(ctx, &p, solver_->solver_kind(), solver_->precision(), saba_order_, 1);
    if (st == ASTER_OK) {
        b.accs.resize(b.positions.size());
        st = aster_state_download(ctx, &b.positions[0].x, &b.velocities[0].x, &b.accs[0].x);
    }
    if (st != ASTER_OK) critical_if(true, std::string("CudaSABA: ") + aster_strerror(st));
}

CudaWH::CudaWH(Simulation* s, CudaSolverBase* solver) : Updater(s, 0, WH_PLANETARY), solver_(solver) {}

void CudaWH::update_bodies() {
    auto& b = _s->bodies;
    if (b.positions.empty()) return;
    if (!uploaded_) {
        solver_->upload();
        uploaded_ = true;
    }
    aster_params p = solver_->params();
    p.force_law = ASTER_NEWTON;
    aster_ctx* ctx = solver_->context();
    int st = aster_wh_steps(ctx, &p, solver_->precision(), 1);
    if (st == ASTER_OK) {
        b.accs.resize(b.positions.size());
        st = aster_state_download(ctx, &b.positions[0].x, &b.velocities[0].x, &b.accs[0].x);
    }
    if (st != ASTER_OK) critical_if(true, std::string("CudaWH: ") + aster_strerror(st));
}

}  // namespace Aster
