// Implementation of the Aster Solver/Updater binding over the C ABI.
#include "aster_cuda_solvers.h"

#include <cstdint>
#include <string>

namespace Aster {

void CudaAllPairs::check(int status, const char* where) {
    if (status == ASTER_OK) return;
    // the reference reports GPU errors through critical_if (logging.cpp:32-47)
    critical_if(true, std::string(where) + ": " + aster_strerror(status));
}

CudaAllPairs::CudaAllPairs(Simulation* s, int precision, int device) : precision_(precision), device_(device) {
    this->_s = s;
    this->type = SIMPLE_GPU;
}

CudaAllPairs::~CudaAllPairs() {
    if (ctx_) aster_ctx_destroy(ctx_);
}

void CudaAllPairs::load() {
    if (!ctx_) check(aster_ctx_create(&ctx_, device_, nullptr), "aster_ctx_create");
}

aster_params CudaAllPairs::params() const {
    aster_params p{};
    p.G = _s->get_G();
    p.c = _s->get_c();
    p.eps2 = _s->softening;
    p.theta = _s->theta;
    p.dt = _s->get_dt();
    p.force_law = force_law.type & (ASTER_NEWTON | ASTER_PN1 | ASTER_PN2 | ASTER_PN25);
    p.morton_bits = 30;
    p.compat_mode = 0;
    p.reserved = 0;
    return p;
}

void CudaAllPairs::upload() {
    load();
    auto& b = _s->bodies;
    const int64_t n = (int64_t)b.positions.size();
    // vec3 is three packed doubles (include/Aster/physics/vectors.h:44-75)
    check(aster_state_upload(ctx_, n, &b.positions[0].x, b.velocities.empty() ? nullptr : &b.velocities[0].x,
                             b.masses.data()),
          "aster_state_upload");
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

CudaLBVH::CudaLBVH(Simulation* s, int precision, int device) : CudaAllPairs(s, precision, device) {
    this->type = GPU_BARNES_HUT;
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
}

// The base Updater is constructed as a leapfrog (a valid entry of
// integrator_mapper, updater.cpp:20-25); update_bodies() replaces it.
CudaKDK::CudaKDK(Simulation* s, CudaAllPairs* solver) : Updater(s, 0, LEAPFROG), solver_(solver) {}

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

CudaSABA::CudaSABA(Simulation* s, CudaAllPairs* solver, int order)
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

CudaWH::CudaWH(Simulation* s, CudaAllPairs* solver) : Updater(s, 0, WH_PLANETARY), solver_(solver) {}

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
