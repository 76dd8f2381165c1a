"""Batched ensemble kernel (C4 setup: hierarchical few-body systems, pairwise
1PN with c = 100, Yoshida-4, dt = 1e-4) against the FP64 CPU oracle, which
uses the reference pair law (compute_gravitational/get_pn1).

Tolerances (max over systems of the relative L2 error of positions and of
velocities after the stated steps): FP64 kernel 1e-9, mixed kernel (FP32 pair
terms on double-single separations) 1e-5. Energies vs the oracle 1e-12.
"""
import threading
import time

import numpy as np
import pytest

from aster_b200 import gen
from aster_b200.api import (EIH, ERR_CANCELLED, FP64, LEAPFROG, MIXED, NEWTON, PN1, PN2, PN25, YOSHIDA4,
                            AsterError, Params)

pytestmark = pytest.mark.gpu

C_LIGHT = 100.0
P = Params(G=1.0, c=C_LIGHT, eps2=0.0, dt=1e-4, force_law=NEWTON | PN1)


def _per_system_err(a, b, off):
    worst = 0.0
    for s in range(len(off) - 1):
        x, y = a[off[s]:off[s + 1]], b[off[s]:off[s + 1]]
        worst = max(worst, np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    return worst


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-9), (MIXED, 1e-5)])
@pytest.mark.parametrize("integrator", [YOSHIDA4, LEAPFROG])
def test_ensemble_vs_oracle(ctx, orc, prec, tol, integrator):
    pos, vel, m, off = gen.hierarchical_ensemble(96, 1004)
    ctx.ensemble_upload(off, pos, vel, m)
    ctx.ensemble_run(P, 50, integrator, prec)
    gp, gv = ctx.ensemble_download()
    op, ov = orc.ens_run(off, pos, vel, m, P.dt, 50, c=C_LIGHT, integrator=integrator)
    assert _per_system_err(gp, op, off) < tol
    assert _per_system_err(gv, ov, off) < tol


def _strong_pn_ensemble():
    """64 softened systems of 2..40 bodies, v ~ 1, eps = 0.1: with c = 10 the
    2PN and 2.5PN terms change the velocities after 20 steps by up to ~10% of
    the total change, far above the tolerances."""
    rng = np.random.default_rng(1007)
    sizes = rng.integers(2, 41, 64)
    off = np.r_[0, np.cumsum(sizes)]
    pos = rng.normal(size=(off[-1], 3))
    vel = rng.normal(size=(off[-1], 3))
    m = rng.uniform(0.5, 1.5, off[-1])
    return pos, vel, m, off


@pytest.mark.parametrize("law", [NEWTON | PN1 | PN2, NEWTON | PN1 | PN25, NEWTON | PN2 | PN25,
                                 NEWTON | PN1 | PN2 | PN25])
def test_higher_pn_ensemble_vs_oracle(ctx, orc, law):
    """get_pn2 / get_pn25 pair terms (the oracle's restatement is pinned to the
    reference in test_oracle.py). FP64 kernel: positions and velocities to
    1e-10. Mixed kernel: the change the 2PN/2.5PN terms make to the state after
    the run (against a run with the same law minus those terms) matches the
    oracle's change to 1e-3 of its size."""
    pos, vel, m, off = _strong_pn_ensemble()
    c, eps2, dt, steps = 10.0, 1e-2, 1e-3, 20
    base = law & ~(PN2 | PN25)

    def run(prec, fl):
        ctx.ensemble_upload(off, pos, vel, m)
        ctx.ensemble_run(Params(G=1.0, c=c, eps2=eps2, dt=dt, force_law=fl), steps, LEAPFROG, prec)
        return ctx.ensemble_download()

    op, ov = orc.ens_run(off, pos, vel, m, dt, steps, c=c, eps2=eps2, integrator=LEAPFROG, pn=law)
    gp, gv = run(FP64, law)
    assert _per_system_err(gp, op, off) < 1e-10
    assert _per_system_err(gv, ov, off) < 1e-10
    bp, bv = orc.ens_run(off, pos, vel, m, dt, steps, c=c, eps2=eps2, integrator=LEAPFROG, pn=base)
    assert np.linalg.norm(ov - bv) > 1e-4 * np.linalg.norm(ov - vel)  # the terms matter
    mp, mv = run(MIXED, law)
    mbp, mbv = run(MIXED, base)
    dv_gpu, dv_orc = mv - mbv, ov - bv
    assert np.linalg.norm(dv_gpu - dv_orc) < 1e-3 * np.linalg.norm(dv_orc)
    assert _per_system_err(mv, ov, off) < 1e-5


def test_post_newtonian_terms_are_rejected_by_the_adjoint(ctx):
    """The adjoint differentiates the Newtonian pair law only: any
    post-Newtonian bit is refused there (every force solver takes them)."""
    pos, vel, m = gen.plummer(256, 3)
    ctx.upload(pos, vel, m)
    for law in (NEWTON | PN1, NEWTON | PN2, NEWTON | PN25):
        p = Params(G=1.0, c=5.0, eps2=1e-3, dt=1e-3, force_law=law)
        with pytest.raises(AsterError) as ei:
            ctx.adjoint(p, 2, pos, FP64, 1)
        assert ei.value.status == 9  # ASTER_ERR_UNSUPPORTED
        assert np.isfinite(ctx.allpairs(p, FP64)).all()
        assert np.isfinite(ctx.lbvh_forces(p, FP64)).all()


def test_higher_pn_ensemble_in_si_units(ctx):
    """Sun-like central masses, AU distances, km/s velocities and the physical
    speed of light: the FP32 post-Newtonian terms stay in range (m_i^2 and
    c^-5 alone would not) and the mixed kernel agrees with FP64."""
    rng = np.random.default_rng(17)
    nsys, k = 64, 4
    off = np.arange(nsys + 1) * k
    au, msun = 1.495978707e11, 1.989e30
    pos = np.zeros((nsys * k, 3))
    vel = np.zeros((nsys * k, 3))
    m = np.zeros(nsys * k)
    for s in range(nsys):
        m[s * k] = msun * rng.uniform(0.5, 2.0)
        for b in range(1, k):
            r = au * rng.uniform(0.05, 2.0)
            ang = rng.uniform(0, 2 * np.pi)
            pos[s * k + b] = [r * np.cos(ang), r * np.sin(ang), 0.0]
            vc = np.sqrt(6.674e-11 * m[s * k] / r)
            vel[s * k + b] = [-vc * np.sin(ang), vc * np.cos(ang), 0.0]
            m[s * k + b] = 6e24 * rng.uniform(0.1, 300.0)
    p = Params(G=6.674e-11, c=299792458.0, eps2=0.0, dt=3600.0, force_law=NEWTON | PN1 | PN2 | PN25)
    out = {}
    for prec in (FP64, MIXED):
        ctx.ensemble_upload(off, pos, vel, m)
        ctx.ensemble_run(p, 24, LEAPFROG, prec)
        out[prec] = ctx.ensemble_download()
    assert np.isfinite(out[MIXED][0]).all() and np.isfinite(out[MIXED][1]).all()
    assert _per_system_err(out[MIXED][0], out[FP64][0], off) < 1e-6


def test_newtonian_ensemble_and_edge_sizes(ctx, orc):
    rng = np.random.default_rng(5)
    sizes = np.array([1, 2, 3, 31, 32, 33, 63, 64, 2, 17])
    off = np.r_[0, np.cumsum(sizes)]
    pos = rng.normal(size=(off[-1], 3))
    vel = rng.normal(size=(off[-1], 3)) * 0.1
    m = rng.uniform(0.5, 1.5, off[-1])
    p = Params(G=1.0, eps2=1e-3, dt=1e-3)
    ctx.ensemble_upload(off, pos, vel, m)
    ctx.ensemble_run(p, 20, YOSHIDA4, FP64)
    gp, gv = ctx.ensemble_download()
    op, ov = orc.ens_run(off, pos, vel, m, p.dt, 20, eps2=1e-3, integrator=YOSHIDA4)
    assert _per_system_err(gp, op, off) < 1e-12
    assert np.allclose(gp[0], pos[0] + 20 * p.dt * vel[0])  # a lone body drifts


def test_oversize_system_rejected(ctx):
    off = np.array([0, 65])
    with pytest.raises(AsterError):
        ctx.ensemble_upload(off, np.zeros((65, 3)), None, np.ones(65))


def test_ensemble_energy_matches_oracle(ctx, orc):
    pos, vel, m, off = gen.hierarchical_ensemble(200, 77)
    ctx.ensemble_upload(off, pos, vel, m)
    e = ctx.ensemble_energy(P)
    eo = orc.ens_energy(off, pos, vel, m, c=C_LIGHT)
    np.testing.assert_allclose(e, eo, rtol=1e-12)


def test_graph_and_plain_launch_agree(ctx):
    pos, vel, m, off = gen.hierarchical_ensemble(300, 9)
    res = []
    for graph in (1, 0):
        ctx.ensemble_upload(off, pos, vel, m)
        ctx.ensemble_run(P, 30, YOSHIDA4, MIXED, {"use_graph": graph, "warps_per_block": 2, "unroll": 4})
        res.append(ctx.ensemble_download()[0])
    np.testing.assert_array_equal(res[0], res[1])  # one warp per system: order-independent


def test_cancel_stops_a_running_kernel(ctx):
    """Failure handling without a GPU fault: a host-written flag polled by
    the persistent kernel ends a long run with ASTER_ERR_CANCELLED."""
    pos, vel, m, off = gen.hierarchical_ensemble(2048, 3)
    ctx.ensemble_upload(off, pos, vel, m)

    def later():
        time.sleep(0.5)
        ctx.ensemble_cancel()

    t = threading.Thread(target=later)
    t0 = time.time()
    t.start()
    with pytest.raises(AsterError) as ei:
        ctx.ensemble_run(P, 2_000_000, YOSHIDA4, MIXED, {"check_every": 64})
    t.join()
    assert ei.value.status == ERR_CANCELLED
    assert time.time() - t0 < 30
    gp, _ = ctx.ensemble_download()
    assert np.isfinite(gp).all()
    # the context stays usable
    ctx.ensemble_upload(off, pos, vel, m)
    ctx.ensemble_run(P, 5, YOSHIDA4, MIXED)


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-9), (MIXED, 1e-5)])
def test_eih_ensemble_vs_oracle(ctx, orc, prec, tol):
    """The N-body Einstein-Infeld-Hoffmann 1PN law (force-law bit EIH) on the
    C4 setup against the oracle's EIH (pinned in test_eih.py to the EIH
    Lagrangian and, for two bodies, to the reference's get_pn1): positions
    and velocities after 50 Yoshida-4 steps per system, FP64 1e-9, mixed
    1e-5; the EIH energy per system 1e-12; and the three-body terms change the
    velocities (against the pairwise law) by 2% of their change over the run
    (asserted > 0.1%), far above either tolerance."""
    pos, vel, m, off = gen.hierarchical_ensemble(96, 1004)
    q = Params(G=1.0, c=C_LIGHT, eps2=0.0, dt=1e-4, force_law=NEWTON | PN1 | EIH)
    ctx.ensemble_upload(off, pos, vel, m)
    e_gpu = ctx.ensemble_energy(q)
    e_orc = orc.ens_energy(off, pos, vel, m, c=C_LIGHT, pn=NEWTON | PN1 | EIH)
    assert np.abs(e_gpu - e_orc).max() <= 1e-12 * np.abs(e_orc).max()
    ctx.ensemble_run(q, 50, YOSHIDA4, prec)
    gp, gv = ctx.ensemble_download()
    op, ov = orc.ens_run(off, pos, vel, m, q.dt, 50, c=C_LIGHT, integrator=YOSHIDA4, pn=NEWTON | PN1 | EIH)
    assert _per_system_err(gp, op, off) < tol
    assert _per_system_err(gv, ov, off) < tol
    pp, pv = orc.ens_run(off, pos, vel, m, q.dt, 50, c=C_LIGHT, integrator=YOSHIDA4, pn=NEWTON | PN1)
    assert np.linalg.norm(ov - pv) > 1e-3 * np.linalg.norm(ov - vel)


def test_eih_strong_field_and_shared_lanes(ctx, orc):
    """EIH where its three-body terms are large (c = 10, softened systems of
    2..40 bodies, v ~ 1; systems above 32 bodies exercise the lanes that split
    a body's sources), leapfrog, 20 steps: FP64 kernel 1e-10, mixed 1e-5."""
    pos, vel, m, off = _strong_pn_ensemble()
    c, eps2, dt, steps = 10.0, 1e-2, 1e-3, 20
    q = Params(G=1.0, c=c, eps2=eps2, dt=dt, force_law=NEWTON | PN1 | EIH)
    ctx.ensemble_upload(off, pos, vel, m)
    ctx.ensemble_run(q, steps, LEAPFROG, FP64)
    gp, gv = ctx.ensemble_download()
    op, ov = orc.ens_run(off, pos, vel, m, dt, steps, c=c, eps2=eps2, integrator=LEAPFROG, pn=NEWTON | PN1 | EIH)
    assert _per_system_err(gp, op, off) < 1e-10
    assert _per_system_err(gv, ov, off) < 1e-10
    ctx.ensemble_upload(off, pos, vel, m)
    ctx.ensemble_run(q, steps, LEAPFROG, MIXED)
    gp, gv = ctx.ensemble_download()
    assert _per_system_err(gp, op, off) < 1e-5
    assert _per_system_err(gv, ov, off) < 1e-5


def test_eih_rejected_outside_ensembles_and_with_higher_orders(ctx):
    pos, vel, m, off = gen.hierarchical_ensemble(8, 5)
    ctx.ensemble_upload(off, pos, vel, m)
    for law in (NEWTON | EIH, NEWTON | PN1 | PN2 | EIH):
        with pytest.raises(AsterError):
            ctx.ensemble_run(Params(c=100.0, force_law=law), 1, YOSHIDA4, FP64)
    ctx.upload(pos, vel, m)
    with pytest.raises(AsterError):
        ctx.allpairs(Params(c=100.0, force_law=NEWTON | PN1 | EIH), FP64)


def test_schedule_leaves_results_unchanged(ctx):
    """Each system is integrated by one warp on its own, so the order in which
    warps take systems (largest first, or upload order) changes nothing: the
    state after the run is bit-identical."""
    pos, vel, m, off = gen.hierarchical_ensemble(512, 1010)
    out = []
    for schedule in (0, 1):
        ctx.ensemble_upload(off, pos, vel, m)
        ctx.ensemble_run(P, 30, YOSHIDA4, MIXED, {"warps_per_block": 4, "unroll": 2, "schedule": schedule})
        out.append(ctx.ensemble_download())
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_autotuner_picks_and_caches(ctx, tmp_path):
    from aster_b200.autotune import tune_ensemble
    pos, vel, m, off = gen.hierarchical_ensemble(1024, 21)
    ctx.ensemble_upload(off, pos, vel, m)
    cache = tmp_path / "tune.json"
    best = tune_ensemble(ctx, off, P, steps=16, space={"warps_per_block": (2, 4), "unroll": (1, 4),
                                                        "schedule": (0, 1)}, cache=cache)
    assert len(best["timings"]) == 8
    # the three fastest short runs were timed again, longer; the best of those wins
    long = [t for t in best["timings"] if "ms_per_step_long" in t]
    assert len(long) == 3
    assert sorted(t["ms_per_step"] for t in long) == sorted(t["ms_per_step"] for t in best["timings"])[:3]
    assert best["ms_per_step_long"] == min(t["ms_per_step_long"] for t in long)
    import torch
    assert best["key"].startswith(torch.cuda.get_device_name(ctx.device) + "|")
    assert cache.exists()
    again = tune_ensemble(ctx, off, P, steps=16, cache=cache)
    assert again["key"] == best["key"]
    gp, _ = ctx.ensemble_download()
    np.testing.assert_array_equal(gp, pos)  # tuning restored the state


def test_c4_full_size_mixed_vs_fp64(ctx):
    """C4 at full size (16384 systems, n in [3, 64]) for 200 steps: mixed vs
    FP64 kernel agree per system (median 1e-8, 99th percentile 1e-4),
    everything finite. The unsoftened e ~ 0.9 inner binaries have pericentre
    passages far shorter than dt = 1e-4; on those few systems any two
    arithmetic paths diverge, so the worst case is not bounded here."""
    pos, vel, m, off = gen.hierarchical_ensemble(16384, 1004)
    out = {}
    for prec in (FP64, MIXED):
        ctx.ensemble_upload(off, pos, vel, m)
        ctx.ensemble_run(P, 200, YOSHIDA4, prec)
        out[prec] = ctx.ensemble_download()[0]
    assert np.isfinite(out[MIXED]).all()
    errs = np.array([np.linalg.norm(out[MIXED][a:b] - out[FP64][a:b]) / np.linalg.norm(out[FP64][a:b])
                     for a, b in zip(off[:-1], off[1:])])
    assert np.median(errs) < 1e-8
    assert np.percentile(errs, 99) < 1e-4


def _c4_sample(nsys=256):
    """The first nsys systems of the C4 ensemble and their measures
    (gen.ensemble_measures: pericentre time, closest other pair, K + |U|)."""
    pos, vel, m, off = gen.hierarchical_ensemble(16384, 1004)
    off = off[:nsys + 1]
    nb = off[-1]
    pos, vel, m = pos[:nb], vel[:nb], m[:nb]
    return (pos, vel, m, off) + gen.ensemble_measures(pos, vel, m, off)


def test_c4_energy_drift_bounds_and_convergence(ctx, orc):
    """C4 drift as evidence: 256 systems of the C4 ensemble, FP64 kernel,
    Yoshida-4 over T = 1 at dt = 1e-4 (the C4 step) and dt/4. Resolved
    systems: inner-binary pericentre time >= 20 dt and no other pair closer
    than 0.5 at the start (109 of 256); the rest have pericentre passages of a
    few steps or close encounters, unsoftened, and no fixed-step integrator
    bounds them. |dE| / (K + |U|) on the resolved systems:
    - Newton only (control): median < 1e-9 at dt (measured 6.6e-11), and the
      drift falls >= 100x at dt/4 (measured 253x: fourth order).
    - EIH 1PN, c = 100: median < 5e-2 at dt (measured 1.4e-2), falling
      >= 2.5x at dt/4 (measured 3.4x): first order, because every kick takes
      the velocity-dependent force at the current velocity, as the
      reference's integrators do.
    - The oracle (FP64 CPU EIH, same composition) on 8 resolved systems of at
      most 16 bodies gives the same energy change to 1% of its size."""
    pos, vel, m, off, tp, dmin, scale = _c4_sample()
    dt = 1e-4
    ok = (tp >= 20 * dt) & (dmin >= 0.5)
    assert ok.sum() >= 80

    def drift(law, step):
        q = Params(G=1.0, c=100.0, eps2=0.0, dt=step, force_law=law)
        ctx.ensemble_upload(off, pos, vel, m)
        e0 = ctx.ensemble_energy(q)
        ctx.ensemble_run(q, int(round(1.0 / step)), YOSHIDA4, FP64)
        return ctx.ensemble_energy(q) - e0

    for law, bound, ratio in ((NEWTON, 1e-9, 100.0), (NEWTON | PN1 | EIH, 5e-2, 2.5)):
        d1, d4 = np.abs(drift(law, dt)) / scale, np.abs(drift(law, dt / 4)) / scale
        assert np.median(d1[ok]) < bound, (law, np.median(d1[ok]))
        assert np.median(d1[ok] / d4[ok]) >= ratio, (law, np.median(d1[ok] / d4[ok]))
    de = drift(NEWTON | PN1 | EIH, dt)
    pick = np.nonzero(ok & (np.diff(off) <= 16))[0][:8]
    assert len(pick) == 8
    for s in pick:
        sl = slice(off[s], off[s + 1])
        sub_off = np.array([0, off[s + 1] - off[s]])
        e0 = orc.ens_energy(sub_off, pos[sl], vel[sl], m[sl], c=100.0, pn=NEWTON | PN1 | EIH)[0]
        p, u = orc.ens_run(sub_off, pos[sl], vel[sl], m[sl], dt, 10_000, c=100.0, integrator=YOSHIDA4,
                           pn=NEWTON | PN1 | EIH)
        de_orc = orc.ens_energy(sub_off, p, u, m[sl], c=100.0, pn=NEWTON | PN1 | EIH)[0] - e0
        assert abs(de[s] - de_orc) <= 1e-2 * abs(de_orc) + 1e-12 * scale[s], (s, de[s], de_orc)


@pytest.mark.parametrize("law", [NEWTON, NEWTON | PN1, NEWTON | PN1 | EIH])
def test_edge_system_sizes_vs_oracle(ctx, orc, law):
    """System sizes at every boundary of the kernel's layout: 1 and 2 bodies,
    odd sizes (a zero-padded half of the last source pair), 31..33 and 63..64
    (the second body per lane), 47..49 (the lanes that split a body's
    sources), softened (eps2 = 1e-2), c = 10, leapfrog, 10 steps: FP64 kernel
    1e-10, mixed 1e-5 against the oracle; a single body moves in a straight
    line."""
    rng = np.random.default_rng(1011)
    sizes = np.array([1, 2, 3, 31, 32, 33, 47, 48, 49, 63, 64, 5, 17])
    off = np.r_[0, np.cumsum(sizes)]
    pos = rng.normal(size=(off[-1], 3))
    vel = rng.normal(size=(off[-1], 3))
    m = rng.uniform(0.5, 1.5, off[-1])
    q = Params(G=1.0, c=10.0, eps2=1e-2, dt=1e-3, force_law=law)
    op, ov = orc.ens_run(off, pos, vel, m, q.dt, 10, c=10.0, eps2=1e-2, integrator=LEAPFROG, pn=law)
    for prec, tol in ((FP64, 1e-10), (MIXED, 1e-5)):
        ctx.ensemble_upload(off, pos, vel, m)
        ctx.ensemble_run(q, 10, LEAPFROG, prec)
        gp, gv = ctx.ensemble_download()
        assert _per_system_err(gp, op, off) < tol, prec
        assert _per_system_err(gv, ov, off) < tol, prec
        np.testing.assert_allclose(gp[0], pos[0] + 10 * q.dt * vel[0], rtol=1e-12)
