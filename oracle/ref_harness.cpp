// C-ABI harness over the reference Aster CPU code, compiled from the reference
// sources unmodified (see oracle/Makefile). TEST INFRASTRUCTURE ONLY: used by
// tests/, the golden-fixture script and bench.py's CPU-baseline leg, never by
// the product.
//
// It drives exactly the reference entry points the hot path replaces:
//   Parallelized::compute_forces   src/utils/builder_endpoint.cpp:729-757
//   Barnes_Hut::make_tree          src/solvers/barnes_hut.cpp:309-400
//   Barnes_Hut::compute_forces     src/solvers/barnes_hut.cpp:402-418
//   get_morton                     src/solvers/bh_specialization.cpp:38-46
//   update_leapfrog                src/physics/tool_chain_impl.cpp:169-185
//   update_SABA1..10               src/integrators/SABA.cpp:14-553 (CPU forms)
//   update_WH_planetary            src/physics/tool_chain_impl.cpp:186-290
//     (also under a zero-force solver: update_kepler, :186-254, on its own)
//   GPU::saba_coeffs               include/Aster/physics/coeffs.h:8-161
//   compute_gravitational          src/physics/tool_chain_impl.cpp:120-137
//   Graphs::get_total_energy       src/utils/collectors.cpp:19-53
//
// One Simulation object lives for the whole process: Parallelized caches the
// first Simulation pointer in a function-static (builder_endpoint.cpp:731),
// so a second Simulation would silently read the first one's bodies.
#include <cstdint>
#include <cstring>
#include <vector>

#include "Aster/simulations/sim_obj.h"
#include "Aster/simulations/barnes-hut.h"
#include "Aster/building-api/builder.h"
#include "Aster/physics/tool-chain.h"
#include "Aster/physics/coeffs.h"
#include "Aster/graphs/graph_collection.h"
#include <tbb/parallel_for.h>

namespace {

// The reference has no setter for G, c or dt as double (set_dt takes float,
// sim_obj.h:99), and `data` is protected, so the harness subclasses it.
struct HarnessSim : public Aster::Simulation {
    void set_consts(double G, double c, double dt) {
        data.G = G;
        data.c = c;
        data.c_squared = c * c;
        data.dt = dt;
    }
};

HarnessSim* g_sim = nullptr;
int g_solver_kind = 0;

// A Solver whose compute_forces() writes zero accelerations. Under it the
// kick of update_WH_planetary does nothing, so one step is two update_kepler
// half-drifts of every body i >= 1 about body 0 (mu = G m_0) plus body 0's
// linear drift: the reference's Kepler drift on its own.
struct ZeroForce : public Aster::Solver {
    explicit ZeroForce(Aster::Simulation* s) { _s = s; }
    void compute_forces() override {
        for (auto& a : _s->bodies.accs) a = Aster::vec3(0.0);
    }
};

HarnessSim* sim() {
    if (!g_sim) g_sim = new HarnessSim();
    return g_sim;
}

}  // namespace

extern "C" {

// solver_kind: 1 = Parallelized (all-pairs), 2 = Barnes_Hut (CPU LBVH).
// force_law: the reference PN bitmask (NEWTON=0x1, PN1=0x10, ...).
// box: half-width of the Morton cube, passed as the screen size so that
// Barnes_Hut::bounding_box = get_center()*2 = (box, box, box).
int ref_setup(int n, const double* pos, const double* vel, const double* mass,
              double G, double c, double dt, double softening, double theta,
              double box, int force_law, int solver_kind) {
    if (n <= 0 || !pos || !vel || !mass) return -1;
    HarnessSim* s = sim();
    s->bodies.positions.resize(n);
    s->bodies.velocities.resize(n);
    s->bodies.accs.assign(n, Aster::vec3(0.0));
    s->bodies.masses.resize(n);
    s->bodies.temps.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        s->bodies.positions[i] = Aster::vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        s->bodies.velocities[i] = Aster::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        s->bodies.masses[i] = mass[i];
    }
    s->set_consts(G, c, dt);
    s->set_screen_size(box, box, box);
    s->softening = softening;
    s->theta = theta;
    s->force_law = Aster::PN_expansion_type((short)force_law);
    s->calculate_total_mass();
    if (s->solver == nullptr || g_solver_kind != solver_kind) {
        delete s->solver;
        s->solver = nullptr;
        if (solver_kind == 1) s->solver = new Aster::Parallelized(s);
        else if (solver_kind == 2) s->solver = new Aster::Barnes::Barnes_Hut(s);
        else return -2;
        g_solver_kind = solver_kind;
    }
    s->solver->force_law = Aster::PN_expansion_type((short)force_law);
    s->solver->set_bounds(0, -1);  // the solver outlives setups: every setup starts with the whole range
    return 0;
}

// Solver::set_bounds (builder_endpoint.cpp:64-67) on the current solver.
int ref_set_bounds(int lower, int upper) {
    HarnessSim* s = sim();
    if (!s->solver) return -1;
    s->solver->set_bounds(lower, upper);
    return 0;
}

int ref_get_state(double* pos, double* vel, double* acc) {
    HarnessSim* s = sim();
    const size_t n = s->bodies.positions.size();
    for (size_t i = 0; i < n; ++i) {
        const auto& p = s->bodies.positions[i];
        const auto& v = s->bodies.velocities[i];
        const auto& a = s->bodies.accs[i];
        if (pos) { pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z; }
        if (vel) { vel[3 * i] = v.x; vel[3 * i + 1] = v.y; vel[3 * i + 2] = v.z; }
        if (acc) { acc[3 * i] = a.x; acc[3 * i + 1] = a.y; acc[3 * i + 2] = a.z; }
    }
    return 0;
}

// One solver->compute_forces() on the current state; accelerations out.
int ref_compute_forces(double* acc_out) {
    HarnessSim* s = sim();
    if (!s->solver) return -1;
    s->solver->compute_forces();
    return ref_get_state(nullptr, nullptr, acc_out);
}

// nsteps of the reference velocity-Verlet leapfrog (2 force evaluations per
// step). acc_steps (nsteps*n*3) receives a(x_{k+1}) after each step if given.
int ref_leapfrog(int nsteps, double* acc_steps) {
    HarnessSim* s = sim();
    if (!s->solver) return -1;
    const size_t n = s->bodies.positions.size();
    for (int k = 0; k < nsteps; ++k) {
        Aster::update_leapfrog(s);
        if (acc_steps) ref_get_state(nullptr, nullptr, acc_steps + (size_t)k * n * 3);
    }
    return 0;
}

// nsteps of the reference CPU SABA_order (order 1..10; SABA1 is update_euler).
int ref_saba(int order, int nsteps) {
    HarnessSim* s = sim();
    if (!s->solver || order < 1 || order > 10) return -1;
    void (*const fns[10])(Aster::Simulation*) = {Aster::update_SABA1, Aster::update_SABA2, Aster::update_SABA3,
                                                 Aster::update_SABA4, Aster::update_SABA5, Aster::update_SABA6,
                                                 Aster::update_SABA7, Aster::update_SABA8, Aster::update_SABA9,
                                                 Aster::update_SABA10};
    for (int k = 0; k < nsteps; ++k) fns[order - 1](s);
    return 0;
}

// The reference's SABA coefficient table for order 1..10, as stored
// ((d, c) slot pairs, d = 0 in the first slot); returns its length.
int ref_saba_coeffs(int order, double* out) {
    if (order < 1 || order > 10) return -1;
    const int len = (int)Aster::GPU::saba_coeff_lng[order - 1];
    for (int i = 0; i < len; ++i) out[i] = Aster::GPU::saba_coeffs[order - 1][i];
    return len;
}

// nsteps of the reference CPU Wisdom-Holman planetary step (body 0 central).
int ref_wh(int nsteps) {
    HarnessSim* s = sim();
    if (!s->solver) return -1;
    for (int k = 0; k < nsteps; ++k) Aster::update_WH_planetary(s);
    return 0;
}

// nsteps of update_WH_planetary with the zero-force solver above in place of
// the current one (restored afterwards): the reference's update_kepler drift
// (tool_chain_impl.cpp:186-254) applied as two half-steps per step.
int ref_wh_drift_only(int nsteps) {
    HarnessSim* s = sim();
    if (s->bodies.positions.empty()) return -1;
    Aster::Solver* keep = s->solver;
    ZeroForce zero(s);
    s->solver = &zero;
    for (int k = 0; k < nsteps; ++k) Aster::update_WH_planetary(s);
    s->solver = keep;
    return 0;
}

double ref_energy() { return Aster::Graphs::get_total_energy(sim()); }

// Builds the CPU LBVH with the reference make_tree and exports it.
// codes[n]: reference get_morton per body (input order).
// left/right[2n-1]: children (-1 = none), leaves 0..n-1, root n.
// node_mass[2n-1], node_com[(2n-1)*3]: after NodesArray::unite.
int ref_bh_tree(uint32_t* codes, int32_t* left, int32_t* right,
                double* node_mass, double* node_com) {
    HarnessSim* s = sim();
    auto* bh = dynamic_cast<Aster::Barnes::Barnes_Hut*>(s->solver);
    if (!bh) return -1;
    bh->make_tree();
    const size_t n = s->bodies.positions.size();
    if (codes)
        for (size_t i = 0; i < n; ++i) codes[i] = Aster::Barnes::get_morton(bh, s->bodies.positions[i]);
    const size_t m = bh->nodes.size();
    if (m != 2 * n - 1) return -2;
    for (size_t i = 0; i < m; ++i) {
        if (left) left[i] = bh->nodes.left_nodes[i];
        if (right) right[i] = bh->nodes.right_nodes[i];
        if (node_mass) node_mass[i] = bh->nodes.masses[i];
        if (node_com) {
            const auto& c = bh->nodes.centers_of_mass[i];
            node_com[3 * i] = c.x; node_com[3 * i + 1] = c.y; node_com[3 * i + 2] = c.z;
        }
    }
    return 0;
}

// Node velocities and temps (NodesArray::unite: mass-weighted mean, maximum)
// of the tree the last ref_bh_tree built; vel[(2n-1)*3], temps[2n-1].
int ref_bh_node_extra(double* vel, double* temps) {
    HarnessSim* s = sim();
    auto* bh = dynamic_cast<Aster::Barnes::Barnes_Hut*>(s->solver);
    if (!bh) return -1;
    const size_t m = bh->nodes.size();
    for (size_t i = 0; i < m; ++i) {
        const auto& v = bh->nodes.velocities[i];
        if (vel) { vel[3 * i] = v.x; vel[3 * i + 1] = v.y; vel[3 * i + 2] = v.z; }
        if (temps) temps[i] = bh->nodes.temps[i];
    }
    return 0;
}

// Body temperatures (BodyArray::temps; ref_setup sets them to 0).
int ref_set_temps(const double* temps) {
    HarnessSim* s = sim();
    for (size_t i = 0; i < s->bodies.temps.size(); ++i) s->bodies.temps[i] = temps[i];
    return 0;
}

// compute_gravitational for one pair (force on body 1, not acceleration),
// with the solver's current force_law.
int ref_pair_force(double m1, double m2, const double* v1, const double* v2,
                   const double* p1, const double* p2, double* f_out) {
    HarnessSim* s = sim();
    if (!s->solver) return -1;
    Aster::vec3 f = Aster::compute_gravitational(
        m1, m2, Aster::vec3(v1[0], v1[1], v1[2]), Aster::vec3(v2[0], v2[1], v2[2]),
        Aster::vec3(p1[0], p1[1], p1[2]), Aster::vec3(p2[0], p2[1], p2[2]), s);
    f_out[0] = f.x; f_out[1] = f.y; f_out[2] = f.z;
    return 0;
}

int ref_threads() { return tbb::shim_threads(); }

}  // extern "C"
