"""SABA_n on the GPU (aster_saba_steps) against the CPU oracle, whose SABA
sequences and coefficients are pinned to the reference's update_SABA1..10
and coefficient table in test_oracle.py.

Tolerances (relative L2 of positions / velocities after the stated steps):
FP64 all-pairs 1e-12; mixed all-pairs (FP32 pair terms on double-single
separations, compensated sums) 1e-7. LBVH (mixed): against the FP64
all-pairs run of the same order, bounded by the theta = 0.5 approximation.
"""
import numpy as np
import pytest

from aster_b200 import api, gen
from aster_b200.api import FP64, MIXED, SOLVER_ALLPAIRS, SOLVER_LBVH, AsterError, Params
from conftest import rel_l2

pytestmark = pytest.mark.gpu

P = Params(G=1.0, eps2=1e-4, dt=1e-3, theta=0.5)


def _state(n=2048, seed=1009):
    return gen.plummer(n, seed)


@pytest.mark.parametrize("order", [1, 2, 3, 4, 6, 10])
def test_saba_fp64_allpairs_vs_oracle(ctx, orc, order):
    pos, vel, m = _state()
    ctx.upload(pos, vel, m)
    ctx.saba_steps(P, order, 5, SOLVER_ALLPAIRS, FP64)
    gp, gv = ctx.download()[:2]
    op, ov = orc.saba(pos, vel, m, P.dt, order, 5, eps2=P.eps2)
    assert rel_l2(gp, op) < 1e-12
    assert rel_l2(gv, ov) < 1e-12


def test_saba_mixed_allpairs_vs_oracle(ctx, orc):
    pos, vel, m = _state()
    ctx.upload(pos, vel, m)
    ctx.saba_steps(P, 4, 5, SOLVER_ALLPAIRS, MIXED)
    gp, gv = ctx.download()[:2]
    op, ov = orc.saba(pos, vel, m, P.dt, 4, 5, eps2=P.eps2)
    assert rel_l2(gp, op) < 1e-7
    assert rel_l2(gv, ov) < 1e-7


def test_saba_lbvh_close_to_allpairs_and_conserves(ctx):
    pos, vel, m = gen.plummer(20000, 1010, masses="lognormal")
    p = Params(G=1.0, eps2=0.005 ** 2, dt=5e-4, theta=0.5)
    ctx.upload(pos, vel, m)
    e0, _ = ctx.energy(p)
    ctx.saba_steps(p, 3, 10, SOLVER_LBVH, MIXED)
    lp, lv = ctx.download()[:2]
    e1, mom = ctx.energy(p)
    ctx.upload(pos, vel, m)
    ctx.saba_steps(p, 3, 10, SOLVER_ALLPAIRS, FP64)
    ap, av = ctx.download()[:2]
    assert rel_l2(lv - vel, av - vel) < 5e-3  # the change of velocity: monopole approximation error
    assert abs(e1 - e0) < 1e-4 * abs(e0)
    assert np.abs(mom).max() < 1e-6


def test_saba_then_kdk_recomputes_acceleration(ctx, orc):
    """SABA leaves no valid cached acceleration (its last drift follows its last
    force evaluation): a following KDK step must evaluate A(x) afresh."""
    pos, vel, m = _state(1024, 1011)
    ctx.upload(pos, vel, m)
    ctx.saba_steps(P, 2, 2, SOLVER_ALLPAIRS, FP64)
    ctx.kdk_steps(P, 1, SOLVER_ALLPAIRS, FP64)
    gp, gv = ctx.download()[:2]
    sp, sv = orc.saba(pos, vel, m, P.dt, 2, 2, eps2=P.eps2)
    op, ov, _, _ = orc.kdk(sp, sv, m, P.dt, 1, eps2=P.eps2)
    assert rel_l2(gp, op) < 1e-12
    assert rel_l2(gv, ov) < 1e-12


@pytest.mark.parametrize("order", [0, 11])
def test_saba_rejects_bad_order(ctx, order):
    pos, vel, m = _state(64, 3)
    ctx.upload(pos, vel, m)
    with pytest.raises(AsterError) as ei:
        ctx.saba_steps(P, order, 1)
    assert ei.value.status == 1  # ASTER_ERR_INVALID_ARG


def test_cuda_saba_updater_in_simulation(orc):
    """The reference-shaped Python mirror: Simulation + CudaAllPairs + CudaSABA."""
    pos, vel, m = _state(1024, 1012)
    sim = api.Simulation(pos, vel, m, G=1.0, dt=1e-3, softening=1e-4)
    sim.solver = api.CudaAllPairs(sim, precision=FP64)
    sim.updater = api.CudaSABA(sim, order=5)
    sim.load()
    for _ in range(3):
        sim.step()
    op, ov = orc.saba(pos, vel, m, 1e-3, 5, 3, eps2=1e-4)
    assert rel_l2(sim.bodies.positions, op) < 1e-12
    assert rel_l2(sim.bodies.velocities, ov) < 1e-12
