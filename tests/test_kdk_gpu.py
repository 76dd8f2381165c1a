"""Fused kick-drift-kick leapfrog (C1: N=4096 Plummer, eps=0.01, dt=1e-3,
100 steps) against the reference's own update_leapfrog trajectory (golden
fixture) and the CPU oracle.

Tolerances: FP64 accelerations/positions 1e-10 relative L2 after up to 100
steps (only rounding differs); mixed 1e-6. Energy drift over 100 steps
|dE/E0| < 1e-6 for both; total momentum stays below 1e-12 (FP64) / 1e-8 (mixed).
"""
import numpy as np
import pytest

from aster_b200 import gen
from aster_b200.api import FP64, MIXED, NEWTON, PN1, PN2, PN25, SOLVER_ALLPAIRS, SOLVER_LBVH, Params
from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-10), (MIXED, 1e-6)])
def test_c1_trajectory_matches_reference(ctx, prec, tol):
    g = golden("leapfrog_plummer4096.npz")
    p = Params(eps2=float(g["eps2"]), dt=float(g["dt"]))
    ctx.upload(g["pos"], g["vel"], g["m"])
    e0, mom0 = ctx.energy(p)
    # the reference's own energy formula, for its own drift number
    er0, _ = ctx.energy(p, ref_form=True)
    assert abs(er0 - float(g["energy0_ref_form"])) < 1e-12 * abs(er0)
    done = 0
    for k, step in enumerate(g["acc_steps"]):
        ctx.kdk_steps(p, int(step) - done, SOLVER_ALLPAIRS, prec)
        done = int(step)
        _, _, acc = ctx.download()
        assert rel_l2(acc, g["acc"][k]) < tol, (step, rel_l2(acc, g["acc"][k]))
    pos, vel, _ = ctx.download()
    assert rel_l2(pos, g["pos_final"]) < tol
    assert rel_l2(vel, g["vel_final"]) < tol
    e1, mom1 = ctx.energy(p)
    assert abs(e1 - e0) / abs(e0) < 1e-6
    assert np.abs(mom1).max() < (1e-12 if prec == FP64 else 1e-8)
    er1, _ = ctx.energy(p, ref_form=True)
    assert abs(er1 - float(g["energy1_ref_form"])) < (1e-10 if prec == FP64 else 1e-7) * abs(er1)


def test_kdk_matches_oracle_kdk(ctx, orc):
    g = golden("leapfrog_plummer4096.npz")
    p = Params(eps2=float(g["eps2"]), dt=float(g["dt"]))
    ctx.upload(g["pos"], g["vel"], g["m"])
    ctx.kdk_steps(p, 5, SOLVER_ALLPAIRS, FP64)
    pos, vel, acc = ctx.download()
    op, ov, oa, _ = orc.kdk(g["pos"], g["vel"], g["m"], p.dt, 5, eps2=p.eps2)
    assert rel_l2(pos, op) < 1e-13
    assert rel_l2(vel, ov) < 1e-12
    assert rel_l2(acc, oa) < 1e-12


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-12), (MIXED, 1e-6)])
def test_kdk_with_every_pn_term_matches_oracle(ctx, orc, prec, tol):
    """KDK on the all-pairs solver with Newton + 1PN + 2PN + 2.5PN (c = 10,
    velocities x5, 5 steps) against the oracle's KDK with the same law."""
    g = golden("allpairs_pn_plummer256.npz")
    law = NEWTON | PN1 | PN2 | PN25
    p = Params(eps2=float(g["eps2"]), dt=1e-3, c=float(g["c"]), force_law=law)
    ctx.upload(g["pos"], g["vel"], g["m"])
    ctx.kdk_steps(p, 5, SOLVER_ALLPAIRS, prec)
    pos, vel, acc = ctx.download()
    op, ov, oa, _ = orc.kdk(g["pos"], g["vel"], g["m"], p.dt, 5, eps2=p.eps2, inv_c=1.0 / p.c, pn=law)
    assert rel_l2(pos, op) < tol
    assert rel_l2(vel, ov) < tol
    assert rel_l2(acc, oa) < tol


def test_energy_matches_oracle(ctx, orc):
    g = golden("leapfrog_plummer4096.npz")
    ctx.upload(g["pos"], g["vel"], g["m"])
    e, mom = ctx.energy(Params(eps2=float(g["eps2"])))
    eo = orc.energy(g["pos"], g["vel"], g["m"], 1.0, float(g["eps2"]))
    assert abs(e - eo) < 1e-12 * abs(eo)
    np.testing.assert_allclose(mom, orc.momentum(g["vel"], g["m"]), atol=1e-15)


def test_simulation_interface(orc):
    """Reference-shaped driver: Simulation + CudaAllPairs + CudaKDK."""
    from aster_b200 import api
    g = golden("leapfrog_plummer4096.npz")
    sim = api.Simulation(g["pos"], g["vel"], g["m"], dt=float(g["dt"]), softening=float(g["eps2"]))
    sim.solver = api.CudaAllPairs(sim)
    sim.updater = api.CudaKDK(sim)
    sim.load()
    sim.solver.compute_forces()
    assert rel_l2(sim.bodies.accs, orc.allpairs(g["pos"], g["m"], 1.0, float(g["eps2"]))) < 1e-12
    sim.step()
    rep = sim.integrate(9, precision_test=True)
    assert rep["precision"] < 1e-7
    assert sim.time_passed == 10
    op, ov, _, _ = orc.kdk(g["pos"], g["vel"], g["m"], float(g["dt"]), 10, eps2=float(g["eps2"]))
    assert rel_l2(sim.bodies.positions, op) < 1e-12


def test_upload_with_accelerations_continues_bit_exactly(ctx):
    """A host round trip of (positions, velocities, accelerations) through
    aster_state_upload_acc continues exactly like the device-resident run (no
    extra force evaluation, same cached acceleration)."""
    from aster_b200.api import Context
    pos, vel, m = gen.plummer(3000, 1021)
    p = Params(G=1.0, eps2=1e-4, dt=1e-3, theta=0.5)
    for solver, prec in ((SOLVER_ALLPAIRS, FP64), (SOLVER_LBVH, MIXED)):
        ctx.upload(pos, vel, m)
        ctx.kdk_steps(p, 3, solver, prec)
        xp, xv, xa = ctx.download()
        with Context(0) as other:
            other.upload(xp, xv, m, acc=xa)
            other.kdk_steps(p, 2, solver, prec)
            op, ov, _ = other.download()
        ctx.kdk_steps(p, 2, solver, prec)
        cp, cv, _ = ctx.download()
        np.testing.assert_array_equal(op, cp)
        np.testing.assert_array_equal(ov, cv)


@pytest.mark.parametrize("prec,law", [(MIXED, NEWTON), (FP64, NEWTON), (MIXED, NEWTON | PN1)])
def test_tree_steps_fused_drift_equal_single_steps(ctx, prec, law):
    """A multi-step tree run applies each next step's opening kick and drift
    inside the previous walk (no kick-drift launch); single-step calls run the
    kick-drift kernel every step. Both give the same state bit for bit."""
    pos, vel, m = gen.plummer(6000, 1030, masses="lognormal")
    p = Params(G=1.0, eps2=0.005 ** 2, dt=5e-4, theta=0.5, c=30.0, force_law=law)
    ctx.upload(pos, vel, m)
    ctx.kdk_steps(p, 6, SOLVER_LBVH, prec)
    fused = ctx.download()
    ctx.upload(pos, vel, m)
    for _ in range(6):
        ctx.kdk_steps(p, 1, SOLVER_LBVH, prec)
    single = ctx.download()
    for a, b in zip(fused, single):
        np.testing.assert_array_equal(a, b)


def test_tree_kdk_graph_kept_across_calls(ctx):
    """The middle steps of a multi-step tree run launch a graph that the
    context keeps from an earlier call with the same parameters, body count
    and buffers. A repeated run (which launches the kept graph) and the first
    run both equal a fresh context's bit for bit; a run with another dt, and
    one with more bodies (the buffers grow), capture anew and equal their own
    fresh-context runs."""
    from aster_b200.api import Context

    def fresh(pos, vel, m, p):
        with Context(0) as other:
            other.upload(pos, vel, m)
            other.kdk_steps(p, 6, SOLVER_LBVH, MIXED)
            return other.download()

    def run(pos, vel, m, p):
        ctx.upload(pos, vel, m)
        ctx.kdk_steps(p, 6, SOLVER_LBVH, MIXED)
        return ctx.download()

    pos, vel, m = gen.plummer(6000, 1031, masses="lognormal")
    p = Params(G=1.0, eps2=0.005 ** 2, dt=5e-4, theta=0.5)
    first, again = run(pos, vel, m, p), run(pos, vel, m, p)
    ref = fresh(pos, vel, m, p)
    for a, b, r in zip(first, again, ref):
        np.testing.assert_array_equal(a, r)
        np.testing.assert_array_equal(b, r)
    p2 = Params(G=1.0, eps2=0.005 ** 2, dt=2.5e-4, theta=0.5)
    for a, r in zip(run(pos, vel, m, p2), fresh(pos, vel, m, p2)):
        np.testing.assert_array_equal(a, r)
    pos3, vel3, m3 = gen.plummer(9000, 1032, masses="lognormal")
    for a, r in zip(run(pos3, vel3, m3, p), fresh(pos3, vel3, m3, p)):
        np.testing.assert_array_equal(a, r)


def test_kdk_steps_host_equals_separate_calls(ctx):
    """aster_kdk_steps_host (one call, the positions' copy overlapping the last
    force evaluation) equals upload_acc + kdk_steps + download bit for bit."""
    from aster_b200.api import Context
    pos, vel, m = gen.plummer(5000, 1022, masses="lognormal")
    p = Params(G=1.0, eps2=0.005 ** 2, dt=5e-4, theta=0.5)
    ctx.upload(pos, vel, m)
    acc0 = ctx.lbvh_forces(p, MIXED)
    for nsteps in (1, 3):
        hp, hv, ha = pos.copy(), vel.copy(), acc0.copy()
        ctx.kdk_steps_host(p, nsteps, hp, hv, ha, m, SOLVER_LBVH, MIXED)
        with Context(0) as other:
            other.upload(pos, vel, m, acc=acc0)
            other.kdk_steps(p, nsteps, SOLVER_LBVH, MIXED)
            op, ov, oa = other.download()
        np.testing.assert_array_equal(hp, op)
        np.testing.assert_array_equal(hv, ov)
        np.testing.assert_array_equal(ha, oa)


def test_c3_disk_long_run_mixed_tracks_fp64():
    """The C3 long run at reduced size: the cold exponential disk (seed of the
    C3 workload) at N = 16384, eps = 0.002, 1000 KDK steps of dt = 1e-4 on
    the all-pairs solver, FP64 and mixed. Energy with the softened potential
    the force derives from (FP64 O(N^2)). Bounds: each drift |dE/E0| < 1e-6
    (measured 1.6e-8 .. 4.4e-8 over the run, a step-size effect common to
    both); mixed minus FP64 drift < 2e-9 (measured 1e-10); final positions
    mixed vs FP64 relative L2 < 1e-8 (measured 5e-10); momentum: FP64
    < 1e-15, mixed < 1e-9 (measured 3e-17 and 6e-11: the FP32 pair terms are
    not exactly antisymmetric). The full-size run (N = 262144) is measured by
    bench.py (allpairs.c3_drift)."""
    from aster_b200.api import Context
    pos, vel, m = gen.exponential_disk(16384, 1003)
    p = Params(G=1.0, eps2=0.002 ** 2, dt=1e-4)
    out = {}
    with Context(0) as c:
        for prec in (FP64, MIXED):
            c.upload(pos, vel, m)
            e0, _ = c.energy(p)
            c.kdk_steps(p, 1000, SOLVER_ALLPAIRS, prec)
            e1, mom = c.energy(p)
            out[prec] = ((e1 - e0) / abs(e0), float(np.abs(mom).max()), c.download()[0])
    d64, mom64, x64 = out[FP64]
    d32, mom32, x32 = out[MIXED]
    assert abs(d64) < 1e-6 and abs(d32) < 1e-6
    assert abs(d32 - d64) < 2e-9, (d32, d64)
    assert rel_l2(x32, x64) < 1e-8
    assert mom64 < 1e-15 and mom32 < 1e-9
    assert rel_l2(x64, pos) > 1e-4  # the disk moved
