"""Device-resident stepping with recorded series (aster_record) against the
same steps taken call by call with a host readback per sample.

The recorded rows use the same kernels in the same order as the call-by-call
path, so energies, momenta and states agree bit for bit; the distance
collector is checked against numpy on the downloaded positions.
"""
import numpy as np
import pytest

from aster_b200 import api, gen
from aster_b200.api import (COLLECT_CENTER, COLLECT_DISTANCE, COLLECT_ENERGY, COLLECT_ENERGY_ERROR,
                            COLLECT_MOMENTUM, FP64, MIXED, SOLVER_ALLPAIRS, SOLVER_LBVH, UPDATER_KDK, UPDATER_SABA,
                            UPDATER_WH, AsterError, Params)
from conftest import rel_l2

pytestmark = pytest.mark.gpu

ALL = COLLECT_ENERGY | COLLECT_ENERGY_ERROR | COLLECT_MOMENTUM | COLLECT_CENTER


@pytest.mark.parametrize("solver,prec", [(SOLVER_ALLPAIRS, FP64), (SOLVER_LBVH, MIXED)])
def test_record_kdk_equals_call_by_call(ctx, solver, prec):
    pos, vel, m = gen.plummer(4096, 1017, masses="lognormal")
    p = Params(G=1.0, eps2=1e-4, dt=1e-3, theta=0.5)
    ctx.upload(pos, vel, m)
    rows, names = ctx.record(p, 30, updater=UPDATER_KDK, solver=solver, precision=prec, rate=5, collect=ALL)
    assert names[:3] == ["time", "energy", "energy_error"] and rows.shape == (7, 1 + 1 + 1 + 3 + 3)
    np.testing.assert_array_equal(rows[:, 0], np.arange(0, 31, 5))
    final = ctx.download()[:2]
    ctx.upload(pos, vel, m)
    e0 = None
    for k in range(7):
        if k:
            ctx.kdk_steps(p, 5, solver, prec)
        e, mom = ctx.energy(p, ref_form=True)
        e0 = e if e0 is None else e0
        assert rows[k, 1] == e
        assert rows[k, 2] == abs(e - e0) / abs(e0)
        np.testing.assert_array_equal(rows[k, 3:6], mom)
    gp, gv = ctx.download()[:2]
    np.testing.assert_array_equal(final[0], gp)
    np.testing.assert_array_equal(final[1], gv)
    com = (m[:, None] * gp).sum(0) / m.sum()
    assert np.abs(rows[-1, 6:9] - com).max() < 1e-13


def test_record_distance_collector(ctx):
    pos, vel, m = gen.plummer(1000, 1018)
    p = Params(G=1.0, eps2=1e-4, dt=1e-3)
    ctx.upload(pos, vel, m)
    rows, names = ctx.record(p, 8, rate=8, collect=COLLECT_DISTANCE)
    assert rows.shape == (2, 1 + 1000) and names[1] == "Body0"
    for k, (xp, _) in enumerate([(pos, None), (ctx.download()[0], None)]):
        com = (m[:, None] * xp).sum(0) / m.sum()
        want = np.linalg.norm(com - xp + 0.1, axis=1)  # distance_collector's offset of 0.1 per component
        assert np.abs(rows[k, 1:] - want).max() < 1e-13


def test_record_tail_steps_and_other_updaters(ctx, orc):
    pos, vel, m = gen.plummer(2048, 1019)
    p = Params(G=1.0, eps2=1e-4, dt=1e-3)
    ctx.upload(pos, vel, m)
    # the Plummer-softened energy is the one this softened force conserves
    rows, _ = ctx.record(p, 7, updater=UPDATER_SABA, order=3, rate=3, collect=COLLECT_ENERGY_ERROR, ref_form=False)
    np.testing.assert_array_equal(rows[:, 0], [0, 3, 6])
    op, ov = orc.saba(pos, vel, m, p.dt, 3, 7, eps2=p.eps2)  # the 7th step is taken too
    gp, gv = ctx.download()[:2]
    assert rel_l2(gp, op) < 1e-12 and rel_l2(gv, ov) < 1e-12
    assert rows[0, 1] == 0.0 and 0 < rows[-1, 1] < 1e-6
    spos, svel, sm = gen.planetary_system(4, 300, 1020)
    ctx.upload(spos, svel, sm)
    rows, _ = ctx.record(Params(G=1.0, dt=0.05), 40, updater=UPDATER_WH, rate=10,
                         collect=COLLECT_ENERGY | COLLECT_ENERGY_ERROR, ref_form=False)
    op, ov = orc.wh(spos, svel, sm, 0.05, 40)
    gp, gv = ctx.download()[:2]
    assert rel_l2(gp, op) < 1e-11 and rel_l2(gv, ov) < 1e-11
    assert rows[-1, 2] < 1e-6  # Wisdom-Holman energy error


def test_record_rejects_bad_config(ctx):
    pos, vel, m = gen.plummer(64, 3)
    ctx.upload(pos, vel, m)
    for kw in ({"rate": 0}, {"collect": 0x100}, {"updater": 7}):
        with pytest.raises(AsterError) as ei:
            ctx.record(Params(dt=1e-3), 4, **kw)
        assert ei.value.status == 1
