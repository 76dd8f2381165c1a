"""The reference-side binding (aster_b200/plugin/aster_cuda_solvers.*) inside
the REFERENCE's own Simulation (compiled from its sources): CudaAllPairs /
CudaLBVH as Aster::Solver and CudaKDK as Aster::Updater, stepped with
Simulation::step(). Compared with the reference's Parallelized solver and
update_leapfrog on the same inputs.

Tolerances: FP64 trajectories 1e-12 relative L2 after 10 steps; PN1
accelerations 1e-12; the LBVH plugin reproduces the C-ABI LBVH bit for bit.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from aster_b200 import gen
from aster_b200.api import FP64, MIXED, NEWTON, PN1, PN2, PN25, SOLVER_LBVH, Params
from conftest import rel_l2

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parent / "plugin" / "_build" / "libaster_plugin_test.so"
_D = ctypes.POINTER(ctypes.c_double)


def _lib():
    if not LIB.exists():
        pytest.skip("plugin harness not built (needs the reference headers at build time)")
    lib = ctypes.CDLL(str(LIB))
    lib.plg_run.argtypes = [ctypes.c_int, _D, _D, _D] + [ctypes.c_double] * 5 + [ctypes.c_int] * 5 + [_D, _D, _D]
    lib.plg_forces_bounds.argtypes = [ctypes.c_int, _D, _D, _D] + [ctypes.c_double] * 3 + [ctypes.c_int] * 5 + [_D]
    return lib


def plugin_run(pos, vel, m, *, G=1.0, c=299792458.0, dt=1e-3, eps2=1e-4, theta=0.5, force_law=NEWTON, solver=0,
               precision=FP64, cuda_kdk=False, nsteps=10, updater=None):
    """updater (overrides cuda_kdk): 0 reference leapfrog, 1 CudaKDK,
    100 + k CudaSABA(k), 200 + k the reference's update_SABAk, 300 CudaWH."""
    lib = _lib()
    n = len(m)
    pos, vel, m = (np.ascontiguousarray(a, dtype=np.float64) for a in (pos, vel, m))
    po, vo, ao = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
    p = lambda a: a.ctypes.data_as(_D)  # noqa: E731
    code = int(cuda_kdk) if updater is None else int(updater)
    rc = lib.plg_run(n, p(pos), p(vel), p(m), G, c, dt, eps2, theta, force_law, solver, precision, code,
                     nsteps, p(po), p(vo), p(ao))
    assert rc == 0
    return po, vo, ao


@pytest.mark.parametrize("cuda_kdk", [False, True])
def test_allpairs_plugin_matches_reference_leapfrog(cuda_kdk):
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference build absent")
    pos, vel, m = gen.plummer(1024, 61)
    po, vo, _ = plugin_run(pos, vel, m, cuda_kdk=cuda_kdk)
    ref = Ref().setup(pos, vel, m, G=1.0, dt=1e-3, eps2=1e-4)
    ref.leapfrog(10)
    rp, rv, _ = ref.state()
    assert rel_l2(po, rp) < 1e-12
    assert rel_l2(vo, rv) < 1e-12


@pytest.mark.parametrize("law", [NEWTON | PN1, NEWTON | PN1 | PN2 | PN25])
def test_pn_through_the_plugin_matches_reference(law):
    """CudaAllPairs reads the Solver's force_law like Parallelized does."""
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference build absent")
    pos, vel, m = gen.plummer(700, 62)
    vel = vel * 30.0
    _, _, ao = plugin_run(pos, vel, m, c=100.0, force_law=law, nsteps=0)
    ref = Ref().setup(pos, vel, m, G=1.0, c=100.0, eps2=1e-4, force_law=law)
    assert rel_l2(ao, ref.forces()) < 1e-12


def test_pn_lbvh_plugin_matches_reference_bh_at_theta0():
    """CudaLBVH with every post-Newtonian term at theta = 0 (every node
    opened) against the reference's Barnes_Hut at theta = 0: both are the full
    pair sum with compute_gravitational."""
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference build absent")
    pos, vel, m = gen.plummer(700, 66)
    vel = vel * 30.0
    law = NEWTON | PN1 | PN2 | PN25
    _, _, ao = plugin_run(pos, vel, m, c=100.0, theta=0.0, force_law=law, solver=1, precision=FP64, nsteps=0)
    ref = Ref().setup(pos, vel, m, G=1.0, c=100.0, eps2=1e-4, theta=0.0, force_law=law, solver="bh")
    assert rel_l2(ao, ref.forces()) < 1e-12


def plugin_forces_bounds(pos, vel, m, lower, upper, *, c=100.0, eps2=1e-4, force_law=NEWTON, solver=0,
                         precision=FP64):
    lib = _lib()
    pos, vel, m = (np.ascontiguousarray(a, dtype=np.float64) for a in (pos, vel, m))
    ao = np.empty((len(m), 3))
    p = lambda a: a.ctypes.data_as(_D)  # noqa: E731
    assert lib.plg_forces_bounds(len(m), p(pos), p(vel), p(m), 1.0, c, eps2, force_law, solver, precision, lower,
                                 upper, p(ao)) == 0
    return ao


@pytest.mark.parametrize("law", [NEWTON, NEWTON | PN1 | PN2 | PN25])
def test_set_bounds_through_the_plugin_matches_parallelized(law):
    """Solver::set_bounds on CudaAllPairs restricts the sources like
    Parallelized (the reference's OpenCL Wisdom-Holman updater sets (1, -1));
    CudaLBVH refuses a range (the reference tree misnumbers its bodies there)
    and leaves the accelerations untouched."""
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference build absent")
    pos, vel, m = gen.plummer(900, 67)
    vel = vel * 30.0
    for lo, hi in ((1, -1), (50, 600)):
        ao = plugin_forces_bounds(pos, vel, m, lo, hi, force_law=law)
        ref = Ref().setup(pos, vel, m, G=1.0, c=100.0, eps2=1e-4, force_law=law).set_bounds(lo, hi).forces()
        assert rel_l2(ao, ref) < 1e-12
    untouched = plugin_forces_bounds(pos, vel, m, 1, -1, force_law=law, solver=1)
    assert np.all(untouched == 1e300)


def test_lbvh_plugin_equals_c_abi(ctx):
    pos, vel, m = gen.plummer(20000, 63, masses="lognormal")
    po, vo, ao = plugin_run(pos, vel, m, eps2=0.005 ** 2, dt=5e-4, solver=1, precision=MIXED, cuda_kdk=True, nsteps=5)
    ctx.upload(pos, vel, m)
    ctx.kdk_steps(Params(eps2=0.005 ** 2, dt=5e-4, theta=0.5), 5, SOLVER_LBVH, MIXED)
    cp, cv, ca = ctx.download()
    np.testing.assert_array_equal(po, cp)
    np.testing.assert_array_equal(vo, cv)


@pytest.mark.parametrize("order", [1, 2, 4, 10])
def test_cuda_saba_plugin_matches_reference_saba_updater(order):
    """The reference's own SABA updater (update_SABAk, driving CudaAllPairs
    FP64 through compute_forces from the host) against CudaSABA (the whole step
    on the device). Order 6 is left out: the reference's update_SABA6 has a
    defective kick slot (see test_oracle.py)."""
    pos, vel, m = gen.plummer(1024, 64)
    ro, rv, _ = plugin_run(pos, vel, m, updater=200 + order, nsteps=3)
    po, pv, _ = plugin_run(pos, vel, m, updater=100 + order, nsteps=3)
    assert rel_l2(po, ro) < 1e-12
    assert rel_l2(pv, rv) < 1e-12
    assert rel_l2(pv, vel) > 1e-4  # the bodies moved


def test_cuda_wh_plugin_matches_oracle(orc):
    """CudaWH inside the reference Simulation: Simulation::step() x 4 equals
    the published Wisdom-Holman method (the oracle)."""
    pos, vel, m = gen.planetary_system(3, 300, 65)
    po, pv, _ = plugin_run(pos, vel, m, dt=0.05, eps2=0.0, updater=300, nsteps=4)
    op, ov = orc.wh(pos, vel, m, 0.05, 4)
    assert rel_l2(po, op) < 1e-12
    assert rel_l2(pv, ov) < 1e-12


def test_lbvh_plugin_is_a_barnes_hut_with_the_reference_tree():
    """CudaLBVH derives from Barnes::Barnes_Hut: with keep_tree, code that
    casts sim->solver to Barnes_Hut* reads the tree of the last evaluation in
    its `nodes`. Against the reference's own make_tree + NodesArray::unite on
    the same bodies (lognormal masses, random temperatures): children, masses
    and centres of mass bit-exact, velocities (mass-weighted) and temps
    (maximum) bit-exact."""
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("reference build absent")
    lib = _lib()
    n = 3000
    pos, vel, m = gen.plummer(n, 4243, masses="lognormal")
    temps = np.random.default_rng(7).uniform(0.0, 100.0, n)
    nm = 2 * n - 1
    mass, com, nvel, ntemp = np.empty(nm), np.empty((nm, 3)), np.empty((nm, 3)), np.empty(nm)
    left, right = np.empty(nm, np.int32), np.empty(nm, np.int32)
    I = ctypes.POINTER(ctypes.c_int32)
    lib.plg_lbvh_tree.argtypes = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_double, ctypes.c_int, _D, _D, _D, _D, I, I]
    p = lambda a: a.ctypes.data_as(_D)  # noqa: E731
    pos, vel, m = (np.ascontiguousarray(a) for a in (pos, vel, m))
    rc = lib.plg_lbvh_tree(n, p(pos), p(vel), p(m), p(temps), 0.5, MIXED, p(mass), p(com), p(nvel), p(ntemp),
                           left.ctypes.data_as(I), right.ctypes.data_as(I))
    assert rc == 0
    B = gen.bounding_cube(pos)
    ref = Ref().setup(pos, vel, m, G=1.0, eps2=1e-4, box=B, solver="bh").set_temps(temps)
    r = ref.bh_tree()
    np.testing.assert_array_equal(left, r["left"])
    np.testing.assert_array_equal(right, r["right"])
    np.testing.assert_array_equal(mass, r["node_mass"])
    np.testing.assert_array_equal(com, r["node_com"])
    np.testing.assert_array_equal(nvel, r["node_vel"])
    np.testing.assert_array_equal(ntemp, r["node_temp"])
