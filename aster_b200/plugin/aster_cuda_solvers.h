// Reference-side binding: Aster Solver/Updater classes backed by the B200
// C ABI (include/aster_cuda.h). A maintainer adds this file and
// aster_cuda_solvers.cpp to Aster's sources and links libaster_cuda.so.
//
//   Solver      include/Aster/simulations/sim_obj.h:34-61
//   Barnes_Hut  include/Aster/simulations/barnes-hut.h:82-117
//   Updater     include/Aster/simulations/sim_obj.h:64-77
//
// Registration (bake_solver, src/utils/updater.cpp:155-170, is a closed
// switch, so the objects are attached after Simulation::load()):
//   sim->load();
//   auto* s = new Aster::CudaLBVH(sim);           // or CudaAllPairs
//   sim->solver = s; s->load();
//   sim->update_with(new Aster::CudaKDK(sim, s)); // optional: device-resident steps
#pragma once

#include "Aster/simulations/barnes-hut.h"
#include "Aster/simulations/sim_obj.h"
#include "aster_cuda.h"

namespace Aster {

// What every B200-backed solver shares, beside its Aster base class: the C-ABI
// context on one device, the precision, and the Simulation's parameters
// (G, c, softening, theta, dt, force law) as aster_params. The updaters below
// drive any solver through this interface.
class CudaSolverBase {
public:
    virtual ~CudaSolverBase();
    aster_ctx* context() const { return ctx_; }
    int precision() const { return precision_; }
    virtual int solver_kind() const = 0;
    aster_params params() const;
    // creates the context on first use
    void ensure_context();
    // copies bodies (positions, velocities, masses) to the device
    void upload();

protected:
    CudaSolverBase(Simulation* s, const Solver* self, int precision, int device)
        : sim_(s), self_(self), precision_(precision), device_(device) {}
    static void check(int status, const char* where);
    Simulation* sim_;
    const Solver* self_;  // the Aster solver object this is part of (its force_law)
    aster_ctx* ctx_ = nullptr;
    int precision_;
    int device_;
};

// Drop-in for Parallelized / SimpleGPU (src/utils/builder_endpoint.cpp:729-757,
// src/solvers/SimpleGPU.cpp:17-71): compute_forces() uploads the bodies,
// evaluates all pairs on the GPU and writes accelerations to bodies.accs,
// honouring force_law (Newton, PN1, PN2, PN2.5), softening, G and c, and the
// source range of Solver::set_bounds.
class CudaAllPairs : public Solver, public CudaSolverBase {
public:
    explicit CudaAllPairs(Simulation* s, int precision = ASTER_MIXED, int device = 0);
    void load() override { ensure_context(); }
    void compute_forces() override;
    int solver_kind() const override { return ASTER_SOLVER_ALLPAIRS; }
};

// Drop-in for Barnes_Hut / BH_hyper (src/solvers/barnes_hut.cpp:402-418,
// src/solvers/full_GPU.cpp:519-527): LBVH build + warp-group walk at
// Simulation::theta; with post-Newtonian bits each accepted node acts with
// its mass-weighted velocity, as Barnes_Hut::get_node_body does. It is a
// Barnes_Hut, so code that casts sim->solver to Barnes::Barnes_Hut* finds
// the tree fields there: after compute_forces() with keep_tree set (or after
// sync_tree()), `nodes` holds the tree of the last evaluation in the
// reference's layout (leaves 0..n-1 = bodies in sorted Morton order, internal
// nodes n..2n-2, root n, -1 = no child; masses and centres of mass as
// NodesArray::unite gives them, velocities mass-weighted and temps the
// children's maximum) and compressed_mortons_size = n.
class CudaLBVH : public Barnes::Barnes_Hut, public CudaSolverBase {
public:
    explicit CudaLBVH(Simulation* s, int precision = ASTER_MIXED, int device = 0);
    void load() override { ensure_context(); }
    void compute_forces() override;
    int solver_kind() const override { return ASTER_SOLVER_LBVH; }
    // rebuilds the tree of the current bodies on the device and copies it into nodes
    void sync_tree();
    bool keep_tree = false;
};

// Drop-in for update_leapfrog (src/physics/tool_chain_impl.cpp:169-185):
// one kick-drift-kick step per update_bodies() with the state kept on the
// device (one force evaluation per step instead of two). bodies.positions /
// velocities / accs are refreshed after every step, since the reference's
// step() only reads GPU buffers back for its own OpenCL solvers.
class CudaKDK : public Updater {
public:
    CudaKDK(Simulation* s, CudaSolverBase* solver);
    void update_bodies() override;
    // next update re-uploads bodies (call after changing them on the host)
    void invalidate() { uploaded_ = false; }

private:
    CudaSolverBase* solver_;
    bool uploaded_ = false;
};

// Drop-in for update_SABA1..10 (src/integrators/SABA.cpp:14-553) and the
// OpenCL SABA updater (src/utils/tc_impl_cl.cpp:269-299): one SABA_order step
// per update_bodies() on the device, order 1..10 (the reference's
// Updater(s, order - 1, SABA) numbering), bodies refreshed after every step.
class CudaSABA : public Updater {
public:
    CudaSABA(Simulation* s, CudaSolverBase* solver, int order);
    void update_bodies() override;
    void invalidate() { uploaded_ = false; }
private:
    CudaSolverBase* solver_;
    int saba_order_;
    bool uploaded_ = false;
};

// Drop-in for update_WH_planetary (src/physics/tool_chain_impl.cpp:186-290)
// and its OpenCL form (include/Aster/kernels/WH_planetary.cl.h): one
// Wisdom-Holman step per update_bodies() with body 0 as the central mass (the
// published democratic heliocentric method; the reference's step re-applies
// the central attraction in its kick). The interaction uses the solver's
// all-pairs kernel at its precision.
class CudaWH : public Updater {
public:
    CudaWH(Simulation* s, CudaSolverBase* solver);
    void update_bodies() override;
    void invalidate() { uploaded_ = false; }
private:
    CudaSolverBase* solver_;
    bool uploaded_ = false;
};

}  // namespace Aster
