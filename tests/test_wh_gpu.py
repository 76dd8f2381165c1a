"""Wisdom-Holman on the GPU (aster_wh_steps) against the FP64 CPU oracle (the
published method in democratic heliocentric coordinates; test_oracle.py shows
why the reference's own step is not the target).

Tolerances (relative L2 of positions / velocities): FP64 1e-11 after 100
steps (the Kepler drifts use the device's sin/cos/sinh/cosh, the oracle the
host's); mixed-precision interaction 3e-8 (FP32 pair terms, ~1e-7 relative,
on an interaction that is ~1e-3 of the acceleration, through 100 steps with
close planet-particle encounters; measured 9e-9).
"""
import numpy as np
import pytest

from aster_b200 import api, gen
from aster_b200.api import FP64, MIXED, AsterError, Params
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _system():
    return gen.planetary_system(6, 4000, 1013)


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-11), (MIXED, 3e-8)])
def test_wh_vs_oracle(ctx, orc, prec, tol):
    pos, vel, m = _system()
    p = Params(G=1.0, eps2=0.0, dt=0.05)
    ctx.upload(pos, vel, m)
    ctx.wh_steps(p, 100, prec)
    gp, gv = ctx.download()[:2]
    op, ov = orc.wh(pos, vel, m, p.dt, 100)
    assert rel_l2(gp, op) < tol
    assert rel_l2(gv, ov) < tol
    assert rel_l2(gv, vel) > 1e-2  # the bodies moved


def test_wh_hyperbolic_and_calls_compose(ctx, orc):
    """A hyperbolic flyby among bound orbits; two calls of 20 steps equal one of 40."""
    pos, vel, m = gen.planetary_system(2, 50, 1014)
    vel[7] = vel[7] * 2.5  # unbound
    p = Params(G=1.0, eps2=1e-6, dt=0.02)
    ctx.upload(pos, vel, m)
    ctx.wh_steps(p, 20)
    ctx.wh_steps(p, 20)
    gp, gv = ctx.download()[:2]
    op, ov = orc.wh(pos, vel, m, p.dt, 40)
    assert rel_l2(gp, op) < 1e-11
    assert rel_l2(gv, ov) < 1e-11


def test_wh_kepler_drift_matches_reference_update_kepler(ctx):
    """The device Kepler drift against the reference's own update_kepler
    (tool_chain_impl.cpp:186-254; golden kepler_drift.npz: update_WH_planetary
    under a zero-force solver on 400 massless bodies about a unit mass,
    elliptic, near-parabolic and hyperbolic orbits, dt = 0.05, 40 steps). With
    only massless bodies a Wisdom-Holman step is one Kepler drift by dt. Per
    body, relative: 1e-11 on elliptic and hyperbolic orbits, 1e-9 near e = 1
    (the device's sin/cos/sinh/cosh against the host's, through 40 drifts)."""
    from conftest import golden
    g = golden("kepler_drift.npz")
    ctx.upload(g["pos"], g["vel"], g["m"])
    ctx.wh_steps(Params(G=1.0, dt=float(g["dt"])), int(g["steps"]), FP64)
    gp, gv = ctx.download()[:2]
    e = g["e"]
    ep = np.linalg.norm(gp[1:] - g["ref_pos"][1:], axis=1) / np.linalg.norm(g["ref_pos"][1:], axis=1)
    ev = np.linalg.norm(gv[1:] - g["ref_vel"][1:], axis=1) / np.linalg.norm(g["ref_vel"][1:], axis=1)
    near = (e > 0.96) & (e < 1.04)
    assert ep[~near].max() < 1e-11 and ev[~near].max() < 1e-11, (ep[~near].max(), ev[~near].max())
    assert ep[near].max() < 1e-9 and ev[near].max() < 1e-9, (ep[near].max(), ev[near].max())


def test_wh_circular_orbit_closes(ctx):
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0]])
    vel = np.array([[0.0, 0, 0], [0, 1.0, 0]])
    m = np.array([1.0, 1e-9])
    ctx.upload(pos, vel, m)
    ctx.wh_steps(Params(G=1.0, dt=2 * np.pi / 200), 200)
    gp, gv = ctx.download()[:2]
    assert np.abs((gp[1] - gp[0]) - [1.0, 0, 0]).max() < 1e-7


def test_wh_errors_leave_context_usable(ctx):
    pos, vel, m = gen.planetary_system(2, 10, 1015)
    p = Params(G=1.0, dt=0.01)
    bad = pos.copy()
    bad[3] = bad[0]  # a body on the central mass: its Kepler drift is undefined
    ctx.upload(bad, vel, m)
    with pytest.raises(AsterError) as ei:
        ctx.wh_steps(p, 2)
    assert ei.value.status == 11  # ASTER_ERR_KEPLER
    assert np.isfinite(ctx.download()[0]).all()
    m0 = m.copy()
    m0[0] = 0.0
    ctx.upload(pos, vel, m0)
    with pytest.raises(AsterError) as ei:
        ctx.wh_steps(p, 1)
    assert ei.value.status == 1  # no positive central mass
    ctx.upload(pos, vel, m)
    ctx.wh_steps(p, 2)
    assert np.isfinite(ctx.download()[0]).all()


def test_cuda_wh_updater_in_simulation(orc):
    pos, vel, m = gen.planetary_system(3, 200, 1016)
    sim = api.Simulation(pos, vel, m, G=1.0, dt=0.05)
    sim.solver = api.CudaAllPairs(sim, precision=FP64)
    sim.updater = api.CudaWH(sim)
    sim.load()
    for _ in range(5):
        sim.step()
    op, ov = orc.wh(pos, vel, m, 0.05, 5)
    assert rel_l2(sim.bodies.positions, op) < 1e-12
    assert rel_l2(sim.bodies.velocities, ov) < 1e-12
