// Test driver for the reference-side binding (aster_b200/plugin): builds a
// reference Aster::Simulation (the reference library compiled from its own
// sources, oracle/_ref), attaches CudaAllPairs / CudaLBVH and either the
// reference's own leapfrog or SABA updater, or CudaKDK / CudaSABA, runs
// Simulation::step() and exports the bodies. TEST INFRASTRUCTURE ONLY.
#include <cstdint>
#include <vector>

#include "Aster/simulations/sim_obj.h"
#include "aster_cuda_solvers.h"

namespace {
// the reference has no double setter for G/c/dt and `data` is protected
struct PluginSim : public Aster::Simulation {
    void set_consts(double G, double c, double dt) {
        data.G = G;
        data.c = c;
        data.c_squared = c * c;
        data.dt = dt;
    }
};
// CudaLBVH (solver_kind 1) is a Barnes::Barnes_Hut, CudaAllPairs a Solver
Aster::Solver* make_solver(Aster::Simulation* s, int solver_kind, int precision) {
    if (solver_kind == 1) return new Aster::CudaLBVH(s, precision);
    return new Aster::CudaAllPairs(s, precision);
}

PluginSim* make_sim(int n, const double* pos, const double* vel, const double* m, const double* temps) {
    auto* s = new PluginSim();
    s->bodies.positions.resize(n);
    s->bodies.velocities.resize(n);
    s->bodies.accs.assign(n, Aster::vec3(0.0));
    s->bodies.masses.assign(m, m + n);
    s->bodies.temps.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        s->bodies.positions[i] = Aster::vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        s->bodies.velocities[i] = Aster::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        if (temps) s->bodies.temps[i] = temps[i];
    }
    return s;
}
}  // namespace

// The tree a CudaLBVH (keep_tree) leaves in the Barnes_Hut fields after one
// compute_forces(), read through a Barnes::Barnes_Hut pointer as reference
// code would: node masses, centres of mass, velocities, temps, children
// (2n - 1 each) and compressed_mortons_size.
extern "C" int plg_lbvh_tree(int n, const double* pos, const double* vel, const double* m, const double* temps,
                             double theta, int precision, double* mass_out, double* com_out, double* vel_out,
                             double* temp_out, int32_t* left_out, int32_t* right_out) {
    if (n <= 0) return -1;
    PluginSim* s = make_sim(n, pos, vel, m, temps);
    s->set_consts(1.0, 299792458.0, 1e-3);
    s->softening = 1e-4;
    s->theta = theta;
    auto* lbvh = new Aster::CudaLBVH(s, precision);
    lbvh->keep_tree = true;
    s->solver = lbvh;
    lbvh->load();
    s->solver->compute_forces();
    auto* bh = dynamic_cast<Aster::Barnes::Barnes_Hut*>(s->solver);
    int rc = 0;
    const size_t mnodes = 2 * (size_t)n - 1;
    if (!bh || bh->nodes.size() != mnodes || bh->compressed_mortons_size != n) {
        rc = -2;
    } else {
        for (size_t i = 0; i < mnodes; ++i) {
            mass_out[i] = bh->nodes.masses[i];
            temp_out[i] = bh->nodes.temps[i];
            left_out[i] = bh->nodes.left_nodes[i];
            right_out[i] = bh->nodes.right_nodes[i];
            const auto& c = bh->nodes.centers_of_mass[i];
            const auto& v = bh->nodes.velocities[i];
            com_out[3 * i] = c.x; com_out[3 * i + 1] = c.y; com_out[3 * i + 2] = c.z;
            vel_out[3 * i] = v.x; vel_out[3 * i + 1] = v.y; vel_out[3 * i + 2] = v.z;
        }
    }
    s->solver = nullptr;
    delete lbvh;
    delete s;
    return rc;
}

// One compute_forces() of CudaAllPairs (solver_kind 0) or CudaLBVH (1) after
// Solver::set_bounds(lower, upper); accelerations out, 1e300 for every body
// whose acceleration the solver did not write (errors go to critical_if).
extern "C" int plg_forces_bounds(int n, const double* pos, const double* vel, const double* m, double G, double c,
                                 double eps2, int force_law, int solver_kind, int precision, int lower, int upper,
                                 double* acc_out) {
    if (n <= 0) return -1;
    auto* s = new PluginSim();
    s->bodies.positions.resize(n);
    s->bodies.velocities.resize(n);
    s->bodies.accs.assign(n, Aster::vec3(0.0));
    s->bodies.masses.assign(m, m + n);
    s->bodies.temps.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        s->bodies.positions[i] = Aster::vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        s->bodies.velocities[i] = Aster::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
    s->set_consts(G, c, 1e-3);
    s->softening = eps2;
    s->force_law = Aster::PN_expansion_type((short)force_law);
    Aster::Solver* solver = make_solver(s, solver_kind, precision);
    solver->force_law = Aster::PN_expansion_type((short)force_law);
    s->solver = solver;
    solver->load();
    solver->set_bounds(lower, upper);
    for (int i = 0; i < n; ++i) s->bodies.accs[i] = Aster::vec3(1e300, 1e300, 1e300);  // marks untouched bodies
    solver->compute_forces();
    for (int i = 0; i < n; ++i) {
        const auto& a = s->bodies.accs[i];
        acc_out[3 * i] = a.x; acc_out[3 * i + 1] = a.y; acc_out[3 * i + 2] = a.z;
    }
    s->solver = nullptr;
    delete solver;
    delete s;
    return 0;
}

extern "C" int plg_run(int n, const double* pos, const double* vel, const double* m, double G, double c, double dt,
                       double eps2, double theta, int force_law, int solver_kind, int precision, int use_cuda_kdk,
                       int nsteps, double* pos_out, double* vel_out, double* acc_out) {
    if (n <= 0) return -1;
    auto* s = new PluginSim();
    s->bodies.positions.resize(n);
    s->bodies.velocities.resize(n);
    s->bodies.accs.assign(n, Aster::vec3(0.0));
    s->bodies.masses.assign(m, m + n);
    s->bodies.temps.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        s->bodies.positions[i] = Aster::vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        s->bodies.velocities[i] = Aster::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
    s->set_consts(G, c, dt);
    s->softening = eps2;
    s->theta = theta;
    s->force_law = Aster::PN_expansion_type((short)force_law);
    Aster::Solver* solver = make_solver(s, solver_kind, precision);
    Aster::CudaSolverBase* base = dynamic_cast<Aster::CudaSolverBase*>(solver);
    solver->force_law = Aster::PN_expansion_type((short)force_law);
    s->solver = solver;
    solver->load();
    // use_cuda_kdk: 0 reference leapfrog, 1 CudaKDK, 100 + k CudaSABA(order k),
    // 200 + k the reference's own SABA updater (update_SABAk) over the solver,
    // 300 CudaWH
    Aster::Updater* up;
    if (use_cuda_kdk == 1) up = new Aster::CudaKDK(s, base);
    else if (use_cuda_kdk > 100 && use_cuda_kdk <= 110) up = new Aster::CudaSABA(s, base, use_cuda_kdk - 100);
    else if (use_cuda_kdk > 200 && use_cuda_kdk <= 210) up = new Aster::Updater(s, use_cuda_kdk - 201, Aster::SABA);
    else if (use_cuda_kdk == 300) up = new Aster::CudaWH(s, base);
    else up = new Aster::Updater(s, 0, Aster::LEAPFROG);
    s->updater = up;
    if (nsteps == 0) solver->compute_forces();
    for (int k = 0; k < nsteps; ++k) s->step();
    for (int i = 0; i < n; ++i) {
        const auto& p = s->bodies.positions[i];
        const auto& v = s->bodies.velocities[i];
        const auto& a = s->bodies.accs[i];
        pos_out[3 * i] = p.x; pos_out[3 * i + 1] = p.y; pos_out[3 * i + 2] = p.z;
        vel_out[3 * i] = v.x; vel_out[3 * i + 1] = v.y; vel_out[3 * i + 2] = v.z;
        acc_out[3 * i] = a.x; acc_out[3 * i + 1] = a.y; acc_out[3 * i + 2] = a.z;
    }
    s->solver = nullptr;
    s->updater = nullptr;
    delete up;
    delete solver;
    delete s;  // never load()ed: the destructor frees nothing else
    return 0;
}
