"""LBVH Barnes-Hut on the GPU against the reference's own tree (golden
fixtures from Barnes_Hut::make_tree) and the CPU oracle.

Bit-exact: Morton codes, sorted order (ties by body index), children,
parents, node ranges, FP64 node masses and centres of mass (NodesArray::unite
order), FP32 bounds and opening radii, per-body interaction-list lengths
(groups = subtrees of <= 64 leaves whose parent holds more).
Forces: FP64 walk vs the oracle's FP64 sum over the same lists 1e-12;
mixed walk 1e-6 (relative L2). Approximation error vs FP64 all-pairs is
reported and bounded (theta = 0.5: < 5e-3; theta = 0: < 1e-12).
"""
import numpy as np
import pytest

from aster_b200 import gen
from aster_b200.api import FP64, MIXED, NEWTON, PN1, PN2, PN25, SOLVER_ALLPAIRS, SOLVER_LBVH, Params
from conftest import golden, rel_l2

pytestmark = pytest.mark.gpu


def _tree_vs_golden(ctx, d):
    ctx.upload(d["pos"], np.zeros_like(d["pos"]), d["m"])
    t = ctx.lbvh_build(Params(theta=0.5))
    assert t["box"] == float(d["box"])
    np.testing.assert_array_equal(t["codes"], d["codes"].astype(np.uint64))
    np.testing.assert_array_equal(t["left"], d["left"])
    np.testing.assert_array_equal(t["right"], d["right"])
    np.testing.assert_array_equal(t["node_mass"], d["node_mass"])
    np.testing.assert_array_equal(t["node_com"], d["node_com"])
    return t


def test_tree_bit_exact_vs_reference(ctx, orc):
    d = golden("tree_plummer4096.npz")
    t = _tree_vs_golden(ctx, d)
    o = orc.lbvh(d["pos"], d["m"], 0.5, B=float(d["box"]))
    for k in ("sorted_codes", "perm", "parent", "range_lo", "range_hi"):
        np.testing.assert_array_equal(t[k], o[k], err_msg=k)
    np.testing.assert_array_equal(t["node_bmin"], o["bmin"])
    np.testing.assert_array_equal(t["node_bmax"], o["bmax"])
    np.testing.assert_array_equal(t["node_rcrit2"], o["rcrit2"])


@pytest.mark.parametrize("case", ["n2", "n3", "n5", "n33", "eq9"])
def test_small_trees_vs_reference(ctx, case):
    d = golden("tree_small.npz")
    _tree_vs_golden(ctx, {k[len(case) + 1:]: d[k] for k in d.files if k.startswith(case + "_")})


def test_single_body(ctx):
    ctx.upload(np.array([[0.5, 0.25, -1.0]]), None, np.array([2.0]))
    acc = ctx.lbvh_forces(Params(eps2=1e-4), MIXED)
    assert np.all(acc == 0)


@pytest.mark.parametrize("bits", [30, 63])
def test_tree_vs_oracle_ragged(ctx, orc, bits):
    for n in (64, 1000, 4097, 70001):
        pos, _, m = gen.plummer(n, 300 + n, masses="lognormal")
        pos[n // 3] = pos[n // 2]
        ctx.upload(pos, None, m)
        t = ctx.lbvh_build(Params(theta=0.5, morton_bits=bits))
        o = orc.lbvh(pos, m, 0.5, bits=bits)
        for k in ("codes", "sorted_codes", "perm", "left", "right", "parent", "range_lo", "range_hi"):
            np.testing.assert_array_equal(t[k], o[k], err_msg=f"{k} n={n}")
        np.testing.assert_array_equal(t["node_com"], o["node_com"])
        np.testing.assert_array_equal(t["node_rcrit2"], o["rcrit2"])


def test_compat_mode_matches_opencl_semantics(ctx, orc):
    """compat_mode = 1: OpenCL gen_mortons (1024 wraps to 0), descending
    (code, index) order, Karras tie-break on body indices; against the oracle
    and, where built, the reference's OpenCL kernels run on the host."""
    pos, _, m = gen.plummer(5000, 88)
    pos[7] = pos[9]
    B = float(np.abs(pos).max())
    ctx.upload(pos, None, m)
    t = ctx.lbvh_build(Params(compat_mode=1))
    codes = orc.morton30(pos, B, compat=True).astype(np.uint64)
    sc, perm = orc.sort_codes(codes, bits=30, descending=True)
    k = orc.karras(sc, perm, bits=30, compat=True)
    np.testing.assert_array_equal(t["codes"], codes)
    np.testing.assert_array_equal(t["perm"], perm)
    np.testing.assert_array_equal(t["left"], k["left"])
    np.testing.assert_array_equal(t["right"], k["right"])
    from oracle.oracle import RefCL
    if RefCL.available():  # the reference's own OpenCL kernels, run on the host
        r = RefCL().build(pos, m, B)
        np.testing.assert_array_equal(t["codes"], r["codes"])
        np.testing.assert_array_equal(t["perm"], r["perm"])
        np.testing.assert_array_equal(t["left"], r["left"])
        np.testing.assert_array_equal(t["right"], r["right"])


@pytest.mark.parametrize("theta", [0.0, 0.3, 0.5, 0.8])
def test_walk_matches_oracle_lists(ctx, orc, theta):
    pos, vel, m = gen.plummer(30000, 1002, masses="lognormal")
    eps2 = 0.005 ** 2
    ctx.upload(pos, vel, m)
    p = Params(eps2=eps2, theta=theta)
    o = orc.lbvh(pos, m, theta)
    oacc, ocnt = orc.lbvh_forces(o, o["perm"], pos, 1.0, eps2)
    a64, c64 = ctx.lbvh_forces(p, FP64, list_counts=True)
    a32, c32 = ctx.lbvh_forces(p, MIXED, list_counts=True)
    np.testing.assert_array_equal(c64, ocnt)
    np.testing.assert_array_equal(c32, ocnt)
    assert rel_l2(a64, oacc) < 1e-12
    assert rel_l2(a32, oacc) < 1e-6
    exact = orc.allpairs(pos, m, 1.0, eps2)
    err = rel_l2(a64, exact)
    bound = {0.0: 1e-12, 0.3: 1e-3, 0.5: 3e-3, 0.8: 1e-2}[theta]  # monopole approximation error
    assert err < bound, err


def test_massless_subtrees_stay_finite_and_cheap(ctx, orc):
    """A massive Plummer sphere and a separate cloud of massless test
    particles: subtrees without mass take the midpoint of their children's
    centres (finite), so they and their ancestors are accepted or opened on
    geometry like any other node. Tree, lists and forces equal the oracle's,
    and a cloud body's list is no longer than a sphere body's several times
    over (a node with no finite centre would be opened down to its leaves)."""
    pos, vel, m = gen.plummer(20000, 1017, masses="lognormal")
    cloud, cvel, _ = gen.plummer(20000, 1018)
    pos2 = np.concatenate([pos, cloud * 0.5 + np.array([3.0, 0.0, 0.0])])
    vel2 = np.concatenate([vel, cvel])
    m2 = np.concatenate([m, np.zeros(20000)])
    eps2 = 0.005 ** 2
    ctx.upload(pos2, vel2, m2)
    t = ctx.lbvh_build(Params(theta=0.5))
    o = orc.lbvh(pos2, m2, 0.5)
    assert np.isfinite(t["node_com"]).all()
    np.testing.assert_array_equal(t["node_mass"], o["node_mass"])
    np.testing.assert_array_equal(t["node_com"], o["node_com"])
    np.testing.assert_array_equal(t["node_rcrit2"], o["rcrit2"])
    oacc, ocnt = orc.lbvh_forces(o, o["perm"], pos2, 1.0, eps2)
    p = Params(eps2=eps2, theta=0.5)
    a64, c64 = ctx.lbvh_forces(p, FP64, list_counts=True)
    a32 = ctx.lbvh_forces(p, MIXED)
    np.testing.assert_array_equal(c64, ocnt)
    assert rel_l2(a64, oacc) < 1e-12
    assert rel_l2(a32, oacc) < 1e-6
    assert ocnt[20000:].mean() < 3 * ocnt[:20000].mean()


@pytest.mark.parametrize("law", [NEWTON | PN1, NEWTON | PN1 | PN2 | PN25])
def test_pn_walk_matches_oracle(ctx, orc, law):
    """Post-Newtonian force law on the tree: as Barnes_Hut::get_node_body,
    every accepted node acts through compute_gravitational with the node's
    mass-weighted velocity (the unite form). Same lists as the oracle's walk;
    forces FP64 1e-12, mixed 1e-6; at theta = 0 (every node opened) the walk
    is the all-pairs sum with the same law."""
    pos, vel, m = gen.plummer(20000, 1019, masses="lognormal")
    vel = vel * 5.0
    c, eps2 = 10.0, 0.005 ** 2
    ctx.upload(pos, vel, m)
    p = Params(eps2=eps2, theta=0.5, c=c, force_law=law)
    o = orc.lbvh(pos, m, 0.5)
    oacc, ocnt = orc.lbvh_forces_pn(o, o["perm"], pos, vel, 1.0, eps2, 1.0 / c, law)
    a64, c64 = ctx.lbvh_forces(p, FP64, list_counts=True)
    a32 = ctx.lbvh_forces(p, MIXED)
    np.testing.assert_array_equal(c64, ocnt)
    assert rel_l2(a64, oacc) < 1e-12
    assert rel_l2(a32, oacc) < 1e-6
    newton, _ = orc.lbvh_forces(o, o["perm"], pos, 1.0, eps2)
    assert rel_l2(oacc, newton) > 1e-3  # the post-Newtonian part is there
    sub = slice(0, 4000)
    ctx.upload(pos[sub], vel[sub], m[sub])
    exact = orc.allpairs(pos[sub], m[sub], 1.0, eps2, vel=vel[sub], inv_c=1.0 / c, pn=law)
    assert rel_l2(ctx.lbvh_forces(Params(eps2=eps2, theta=0.0, c=c, force_law=law), FP64), exact) < 1e-12


def test_pn_lbvh_kdk_at_theta0_equals_allpairs_kdk(ctx):
    """KDK on the tree with every post-Newtonian term (closing kick fused
    into the walk, node velocities rebuilt each step from the half-kicked
    velocities) at theta = 0 equals KDK on the all-pairs solver: FP64 1e-12,
    mixed tree vs FP64 all-pairs 1e-6."""
    pos, vel, m = gen.plummer(4096, 1020)
    vel = vel * 5.0
    p = Params(eps2=1e-4, dt=1e-3, theta=0.0, c=10.0, force_law=NEWTON | PN1 | PN2 | PN25)
    out = {}
    for solver, prec in ((SOLVER_LBVH, FP64), (SOLVER_LBVH, MIXED), (SOLVER_ALLPAIRS, FP64)):
        ctx.upload(pos, vel, m)
        ctx.kdk_steps(p, 3, solver, prec)
        out[(solver, prec)] = ctx.download()
    ref = out[(SOLVER_ALLPAIRS, FP64)]
    for key, tol in (((SOLVER_LBVH, FP64), 1e-12), ((SOLVER_LBVH, MIXED), 1e-6)):
        for k in range(3):
            assert rel_l2(out[key][k], ref[k]) < tol, (key, k)


def test_zero_softening_walk_is_finite(ctx):
    """eps = 0 with two coincident bodies: the zero separations contribute
    nothing (Newton, and Newton + 1PN, whose mixed walk pairs list entries)."""
    pos, vel, m = gen.plummer(5000, 3)
    pos[1] = pos[2]
    ctx.upload(pos, vel, m)
    for law in (NEWTON, NEWTON | PN1):
        for prec in (FP64, MIXED):
            assert np.isfinite(ctx.lbvh_forces(Params(eps2=0.0, c=10.0, force_law=law), prec)).all()


def test_c2_full_size_tree_bit_exact(ctx, orc):
    """C2 at full size (n = 2^20, lognormal Plummer): the whole tree equals the
    CPU restatement (itself pinned bit-exact to the reference above)."""
    n = 1 << 20
    pos, vel, m = gen.plummer(n, 1002, masses="lognormal")
    ctx.upload(pos, vel, m)
    t = ctx.lbvh_build(Params(theta=0.5, eps2=0.005 ** 2))
    o = orc.lbvh(pos, m, 0.5)
    for k in ("codes", "sorted_codes", "perm", "left", "right", "parent", "range_lo", "range_hi"):
        np.testing.assert_array_equal(t[k], o[k], err_msg=k)
    np.testing.assert_array_equal(t["node_mass"], o["node_mass"])
    np.testing.assert_array_equal(t["node_com"], o["node_com"])
    np.testing.assert_array_equal(t["node_rcrit2"], o["rcrit2"])
    sc = t["sorted_codes"]
    assert np.all(sc[1:] >= sc[:-1])
    ties = sc[1:] == sc[:-1]
    assert np.all(t["perm"][1:][ties] > t["perm"][:-1][ties])


def test_c2_full_size_tree_bit_exact_vs_reference_build(ctx):
    """C2 at full size against the reference itself: Barnes_Hut::make_tree
    (src/solvers/barnes_hut.cpp:309-400, unite :137-152) run by the reference
    CPU library on the same 2^20 bodies and Morton box. Morton codes, left and
    right children of every node, FP64 node masses and centres of mass are
    bit-identical; the leaves hold the bodies in our sorted order (the
    reference stores each sorted body's position and mass in leaf i)."""
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference CPU build absent")
    n = 1 << 20
    pos, vel, m = gen.plummer(n, 1002, masses="lognormal")
    ctx.upload(pos, vel, m)
    t = ctx.lbvh_build(Params(theta=0.5, eps2=0.005 ** 2))
    ref = Ref().setup(pos, vel, m, G=1.0, eps2=0.005 ** 2, theta=0.5, box=t["box"], solver="bh")
    r = ref.bh_tree()
    np.testing.assert_array_equal(t["codes"], r["codes"].astype(np.uint64))
    np.testing.assert_array_equal(t["left"], r["left"])
    np.testing.assert_array_equal(t["right"], r["right"])
    np.testing.assert_array_equal(t["node_mass"], r["node_mass"])
    np.testing.assert_array_equal(t["node_com"], r["node_com"])
    np.testing.assert_array_equal(pos[t["perm"]], r["node_com"][:n])
    np.testing.assert_array_equal(m[t["perm"]], r["node_mass"][:n])


def test_c2_full_size_forces_sampled(ctx):
    """C2 forces at full size: mixed vs FP64 walk on every body (same lists),
    approximation error vs FP64 all-pairs on a fixed 4096-body sample."""
    n = 1 << 20
    pos, vel, m = gen.plummer(n, 1002, masses="lognormal")
    ctx.upload(pos, vel, m)
    p = Params(theta=0.5, eps2=0.005 ** 2)
    a32 = ctx.lbvh_forces(p, MIXED)
    a64 = ctx.lbvh_forces(p, FP64)
    assert rel_l2(a32, a64) < 1e-6
    tg = np.random.default_rng(4096).choice(n, 4096, replace=False)
    exact = ctx.allpairs_targets(p, tg, FP64)
    err = rel_l2(a32[tg], exact)
    assert err < 5e-3, err


def test_walk_stack_overflow_is_reported(monkeypatch):
    """Failure path without a GPU fault: a tiny usable stack (host-side limit,
    the shared-memory stack is unchanged) makes the walk stop early and the
    call return ASTER_ERR_STACK; the context and the GPU stay usable."""
    from aster_b200.api import AsterError, Context
    pos, vel, m = gen.plummer(5000, 12)
    monkeypatch.setenv("ASTER_WALK_STACK_LIMIT", "64")
    with Context(0) as small:
        small.upload(pos, vel, m)
        with pytest.raises(AsterError) as ei:
            small.lbvh_forces(Params(eps2=1e-4, theta=0.0), MIXED)
        assert ei.value.status == 5  # ASTER_ERR_STACK
        assert np.isfinite(small.allpairs(Params(eps2=1e-4), FP64)).all()
    monkeypatch.delenv("ASTER_WALK_STACK_LIMIT")
    with Context(0) as normal:
        normal.upload(pos, vel, m)
        assert np.isfinite(normal.lbvh_forces(Params(eps2=1e-4, theta=0.0), MIXED)).all()


def test_lbvh_kdk_conserves(ctx):
    pos, vel, m = gen.plummer(50000, 1002, masses="lognormal")
    ctx.upload(pos, vel, m)
    p = Params(theta=0.5, eps2=0.005 ** 2, dt=5e-4)
    e0, _ = ctx.energy(p)
    ctx.kdk_steps(p, 10, SOLVER_LBVH, MIXED)
    e1, mom = ctx.energy(p)
    assert abs(e1 - e0) / abs(e0) < 1e-4
    assert np.abs(mom).max() < 1e-6
