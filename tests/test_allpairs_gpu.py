"""All-pairs force kernels (FP64 and mixed) against the reference's own
accelerations (golden fixtures) and the CPU oracle, through the C ABI.

Tolerances (relative L2 over all components, stated per test):
  FP64 vs reference/oracle       1e-12
  mixed (FP32 pairs, compensated) vs FP64 oracle   1e-6
"""
import numpy as np
import pytest

from aster_b200 import gen
from aster_b200.api import FP64, MIXED, NEWTON, PN1, PN2, PN25, Params
from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-6


def test_fp64_matches_reference_golden(ctx):
    g = golden("allpairs_plummer512.npz")
    ctx.upload(g["pos"], g["vel"], g["m"])
    a = ctx.allpairs(Params(eps2=float(g["eps2"])), FP64)
    assert rel_l2(a, g["acc"]) < TOL_FP64


def test_mixed_matches_reference_golden(ctx):
    g = golden("allpairs_plummer512.npz")
    ctx.upload(g["pos"], g["vel"], g["m"])
    a = ctx.allpairs(Params(eps2=float(g["eps2"])), MIXED)
    assert rel_l2(a, g["acc"]) < TOL_MIXED


@pytest.mark.parametrize("prec,tol", [(FP64, TOL_FP64), (MIXED, TOL_MIXED)])
def test_pn1_matches_reference_golden(ctx, prec, tol):
    g = golden("allpairs_plummer512.npz")
    ctx.upload(g["pos"], g["vel_pn"], g["m"])
    p = Params(eps2=float(g["eps2"]), c=float(g["c_pn"]), force_law=NEWTON | PN1)
    a = ctx.allpairs(p, prec)
    assert rel_l2(a, g["acc_pn1"]) < tol
    # the PN part alone (acc_pn1 - newton) to 1e-4 relative in mixed precision
    newton = golden("allpairs_plummer512.npz")["acc"]
    assert rel_l2(a - newton, g["acc_pn1"] - newton) < (1e-10 if prec == FP64 else 1e-3)


PN_LAWS = {"pn1": NEWTON | PN1, "pn2": NEWTON | PN2, "pn25": NEWTON | PN25, "all": NEWTON | PN1 | PN2 | PN25}


@pytest.mark.parametrize("name", list(PN_LAWS))
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_pn_laws_match_reference_golden(ctx, name, prec):
    """Parallelized::compute_forces with each post-Newtonian force law (N = 256,
    c = 10; the 1PN, 2PN and 2.5PN parts are 0.15, 0.02 and 3e-5 of the
    Newtonian sum). Total: FP64 1e-12, mixed 1e-6. Post-Newtonian part (law
    minus the reference's Newtonian accelerations), as an absolute L2 bound:
    FP64 1e-13 |Newton| + 1e-10 |part|; mixed 2e-7 |Newton| (the Newtonian
    sum's own error) + 1e-5 |part| (FP32 post-Newtonian sums)."""
    g = golden("allpairs_pn_plummer256.npz")
    ctx.upload(g["pos"], g["vel"], g["m"])
    p = Params(eps2=float(g["eps2"]), c=float(g["c"]), force_law=PN_LAWS[name])
    a = ctx.allpairs(p, prec)
    ref, newton = g[f"acc_{name}"], g["acc_newton"]
    assert rel_l2(a, ref) < (1e-12 if prec == FP64 else 1e-6)
    part = ref - newton
    bound = (1e-13 * np.linalg.norm(newton) + 1e-10 * np.linalg.norm(part) if prec == FP64
             else 2e-7 * np.linalg.norm(newton) + 1e-5 * np.linalg.norm(part))
    assert np.linalg.norm((a - newton) - part) < bound


@pytest.mark.parametrize("law", [NEWTON, NEWTON | PN1 | PN2 | PN25])
def test_source_range_matches_reference_set_bounds(ctx, law):
    """aster_allpairs_range against Parallelized::compute_forces after
    Solver::set_bounds(lower, upper): every body gets the pull of the sources
    [lower, upper) only (FP64 1e-12, mixed 1e-6); an empty range gives zeros."""
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference build absent")
    pos, vel, m = gen.plummer(1500, 71)
    vel = vel * 30.0
    p = Params(eps2=1e-4, c=100.0, force_law=law)
    ctx.upload(pos, vel, m)
    for lo, hi in ((1, -1), (100, 900), (0, 1500), (1499, 1500)):
        ref = Ref().setup(pos, vel, m, G=1.0, c=100.0, eps2=1e-4, force_law=law).set_bounds(lo, hi).forces()
        assert rel_l2(ctx.allpairs_range(p, lo, hi, FP64), ref) < 1e-12, (lo, hi)
        assert rel_l2(ctx.allpairs_range(p, lo, hi, MIXED), ref) < 1e-6, (lo, hi)
    assert np.all(ctx.allpairs_range(p, 700, 700, FP64) == 0.0)
    full = ctx.allpairs(p, FP64)
    assert rel_l2(ctx.allpairs_range(p, 0, -1, FP64), full) == 0.0


def test_pn_laws_in_si_units(ctx, orc):
    """A star of 2e30 kg with 500 planets and planetesimals at 0.05-5 AU on
    near-circular orbits, SI units, physical c, every PN term: FP64 equals the
    oracle to 1e-12 and the mixed kernel (FP32 post-Newtonian sums, written so
    that m^2 and c^-5 never appear alone) stays finite and within 1e-6."""
    rng = np.random.default_rng(23)
    n = 501
    G, msun, au = 6.674e-11, 2.0e30, 1.495978707e11
    r = au * np.exp(rng.uniform(np.log(0.05), np.log(5.0), n - 1))
    ang = rng.uniform(0, 2 * np.pi, n - 1)
    pos = np.zeros((n, 3))
    vel = np.zeros((n, 3))
    pos[1:, 0], pos[1:, 1] = r * np.cos(ang), r * np.sin(ang)
    pos[1:, 2] = r * rng.normal(0, 0.01, n - 1)
    vc = np.sqrt(G * msun / r)
    vel[1:, 0], vel[1:, 1] = -vc * np.sin(ang), vc * np.cos(ang)
    m = np.r_[msun, 6e24 * np.exp(rng.uniform(np.log(1e-3), np.log(300.0), n - 1))]
    law = NEWTON | PN1 | PN2 | PN25
    p = Params(G=G, c=299792458.0, eps2=0.0, force_law=law)
    ctx.upload(pos, vel, m)
    ref = orc.allpairs(pos, m, G, 0.0, vel=vel, inv_c=1.0 / 299792458.0, pn=law)
    a64 = ctx.allpairs(p, FP64)
    a32 = ctx.allpairs(p, MIXED)
    assert rel_l2(a64, ref) < 1e-12
    assert np.isfinite(a32).all()
    assert rel_l2(a32, ref) < 1e-6


@pytest.mark.parametrize("n", [1, 2, 3, 31, 33, 127, 129, 1000, 4097])
def test_ragged_sizes_vs_oracle(ctx, orc, n):
    pos, vel, m = gen.plummer(n, 500 + n) if n > 1 else (np.array([[0.3, -0.2, 0.1]]), np.zeros((1, 3)), np.ones(1))
    ctx.upload(pos, vel, m)
    p = Params(eps2=1e-4)
    ref = orc.allpairs(pos, m, 1.0, 1e-4)
    a64 = ctx.allpairs(p, FP64)
    a32 = ctx.allpairs(p, MIXED)
    if n == 1:
        assert np.all(a64 == 0) and np.all(a32 == 0)
        return
    assert rel_l2(a64, ref) < TOL_FP64
    assert rel_l2(a32, ref) < TOL_MIXED


def test_zero_softening_coincident_bodies(ctx):
    """eps2 = 0 with exact duplicates: zero-distance pairs are skipped (the
    reference would divide by zero); every other pair is exact."""
    pos, vel, m = gen.plummer(300, 9)
    pos[10] = pos[20]
    pos[11] = pos[20]
    ctx.upload(pos, vel, m)
    d = pos[None, :, :] - pos[:, None, :]
    r2 = (d ** 2).sum(-1)
    with np.errstate(divide="ignore"):
        w = np.where(r2 > 0, r2 ** -1.5, 0.0)
    ref = (d * (m[None, :, None] * w[:, :, None])).sum(1)
    for prec, tol in ((FP64, TOL_FP64), (MIXED, TOL_MIXED)):
        a = ctx.allpairs(Params(eps2=0.0), prec)
        assert np.isfinite(a).all()
        assert rel_l2(a, ref) < tol


def test_targets_api(ctx, orc):
    pos, vel, m = gen.plummer(20000, 31, masses="lognormal")
    ctx.upload(pos, vel, m)
    tg = np.random.default_rng(1).choice(20000, 300, replace=False).astype(np.int32)
    ref = orc.allpairs(pos, m, 1.0, 2.5e-5, targets=tg)
    p = Params(eps2=2.5e-5)
    assert rel_l2(ctx.allpairs_targets(p, tg, FP64), ref) < TOL_FP64
    assert rel_l2(ctx.allpairs_targets(p, tg, MIXED), ref) < TOL_MIXED


def test_disk_mixed_precision_small(ctx, orc):
    """Cold disk with eps = 0.002 (C3 setup at n = 16384): close pairs far
    from the origin are where plain FP32 positions would fail."""
    pos, vel, m = gen.exponential_disk(16384, 1003)
    ctx.upload(pos, vel, m)
    p = Params(eps2=0.002 ** 2)
    ref = orc.allpairs(pos, m, 1.0, p.eps2)
    assert rel_l2(ctx.allpairs(p, FP64), ref) < TOL_FP64
    assert rel_l2(ctx.allpairs(p, MIXED), ref) < TOL_MIXED


def test_disk_full_size_sampled(ctx, orc):
    """C3 at full size (n = 262144): mixed vs FP64 on every body, and both
    against the CPU oracle on 256 sampled targets."""
    pos, vel, m = gen.exponential_disk(262144, 1003)
    ctx.upload(pos, vel, m)
    p = Params(eps2=0.002 ** 2)
    a64 = ctx.allpairs(p, FP64)
    a32 = ctx.allpairs(p, MIXED)
    assert rel_l2(a32, a64) < TOL_MIXED
    tg = np.random.default_rng(3).choice(262144, 256, replace=False)
    ref = orc.allpairs(pos, m, 1.0, p.eps2, targets=tg)
    assert rel_l2(a64[tg], ref) < TOL_FP64
    assert rel_l2(a32[tg], ref) < TOL_MIXED


def test_invalid_arguments(ctx):
    from aster_b200.api import AsterError
    ctx.upload(*gen.plummer(64, 1))
    with pytest.raises(AsterError):
        ctx.allpairs(Params(eps2=-1.0), FP64)
    with pytest.raises(AsterError):
        ctx.allpairs(Params(), 7)
    with pytest.raises(AsterError):
        ctx.upload(np.array([[np.nan, 0, 0]]), None, np.ones(1))


def test_empty_input_and_missing_state():
    """A context with no bodies answers every solver, stepper and readback
    with ASTER_ERR_NO_STATE and stays usable; an empty body array is an
    invalid argument and leaves the context without state (the C++ plugin
    returns early for an empty body array, as the reference's solvers do)."""
    from aster_b200.api import SOLVER_LBVH, AsterError, Context
    with Context(0) as c:
        calls = (lambda: c.allpairs(Params(), FP64), lambda: c.allpairs(Params(), MIXED),
                 lambda: c.lbvh_forces(Params()), lambda: c.kdk_steps(Params(), 1),
                 lambda: c.kdk_steps(Params(), 1, SOLVER_LBVH, MIXED), lambda: c.energy(Params()),
                 lambda: c.download())
        for call in calls:
            with pytest.raises(AsterError) as e:
                call()
            assert e.value.status == 4  # ASTER_ERR_NO_STATE
        with pytest.raises(AsterError) as e:
            c.upload(np.zeros((0, 3)), None, np.zeros(0))
        assert e.value.status == 1  # ASTER_ERR_INVALID_ARG
        with pytest.raises(AsterError) as e:
            c.allpairs(Params(), FP64)
        assert e.value.status == 4
        # above the largest supported n (2^30: node ids are int32) the size is
        # refused before any pointer is read
        pos, vel, m = gen.plummer(100, 5)
        too_many = c.lib.aster_state_upload(c.h, (1 << 30) + 1, pos.ctypes.data, vel.ctypes.data, m.ctypes.data)
        assert too_many == 1  # ASTER_ERR_INVALID_ARG
        c.upload(pos, vel, m)
        assert np.all(np.isfinite(c.allpairs(Params(eps2=1e-4), FP64)))


@pytest.mark.parametrize("n_massive", [1, 5, 700])
def test_trailing_massless_sources(ctx, orc, n_massive):
    """Bodies after the last massive one are skipped as sources (they attract
    nothing); results equal the oracle's sum over every body, for Newton and
    1PN, all targets and a target list, and a later upload with massive tail
    bodies uses them again."""
    n = 3000
    pos, vel, m = gen.plummer(n, 77 + n_massive)
    vel = vel * 0.1
    m0 = m.copy()
    m[n_massive:] = 0.0
    if n_massive > 2:
        m[n_massive // 2] = 0.0  # a massless body before the last massive one
    ctx.upload(pos, vel, m)
    for law, cval in ((NEWTON, 0.0), (NEWTON | PN1, 30.0)):
        p = Params(eps2=1e-4, c=cval, force_law=law)
        ref = orc.allpairs(pos, m, 1.0, 1e-4, vel=vel, inv_c=1.0 / cval if cval else 0.0, pn=law)
        assert rel_l2(ctx.allpairs(p, FP64), ref) < TOL_FP64
        assert rel_l2(ctx.allpairs(p, MIXED), ref) < TOL_MIXED
    tg = np.arange(n - 200, n, dtype=np.int32)
    ref = orc.allpairs(pos, m, 1.0, 1e-4, targets=tg)
    assert rel_l2(ctx.allpairs_targets(Params(eps2=1e-4), tg, MIXED), ref) < TOL_MIXED
    ctx.upload(pos, vel, m0)
    ref = orc.allpairs(pos, m0, 1.0, 1e-4)
    assert rel_l2(ctx.allpairs(Params(eps2=1e-4), FP64), ref) < TOL_FP64


def test_mixed_allpairs_sees_the_state_left_by_other_steppers(ctx):
    """A mixed all-pairs evaluation after steps taken another way (tree KDK,
    FP64 all-pairs KDK, SABA, mixed KDK whose closing kick moved the
    velocities) uses the current positions and velocities: it agrees with the
    FP64 evaluation of the same state, Newtonian and 1PN."""
    from aster_b200.api import SOLVER_ALLPAIRS, SOLVER_LBVH
    pos, vel, m = gen.plummer(4096, 91)
    step = Params(eps2=1e-4, dt=5e-3, c=30.0, force_law=NEWTON | PN1)
    steppers = {
        "lbvh_fp64": lambda: ctx.kdk_steps(Params(eps2=1e-4, dt=5e-3), 3, SOLVER_LBVH, FP64),
        "allpairs_fp64": lambda: ctx.kdk_steps(step, 3, SOLVER_ALLPAIRS, FP64),
        "allpairs_mixed_pn": lambda: ctx.kdk_steps(step, 3, SOLVER_ALLPAIRS, MIXED),
        "saba2_fp64": lambda: ctx.saba_steps(step, 2, 2, SOLVER_ALLPAIRS, FP64),
    }
    for name, run in steppers.items():
        ctx.upload(pos, vel * 3.0, m)
        run()
        for law in (NEWTON, NEWTON | PN1):
            q = Params(eps2=1e-4, c=30.0, force_law=law)
            a64 = ctx.allpairs(q, FP64)
            a32 = ctx.allpairs(q, MIXED)
            assert rel_l2(a32, a64) < TOL_MIXED, (name, law)
