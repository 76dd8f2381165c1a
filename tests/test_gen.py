"""Seeded generators: determinism and the stated distribution properties."""
import numpy as np

from aster_b200 import gen


def test_plummer_deterministic_and_centred():
    a = gen.plummer(4096, 1001)
    b = gen.plummer(4096, 1001)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    pos, vel, m = a
    assert abs(m.sum() - 1.0) < 1e-12
    np.testing.assert_allclose((m[:, None] * pos).sum(0), 0, atol=1e-14)
    np.testing.assert_allclose((m[:, None] * vel).sum(0), 0, atol=1e-14)
    r = np.linalg.norm(pos, axis=1)
    assert r.max() < 10.5
    # half-mass radius of a Plummer sphere ~ 1.305 a (truncation shifts it slightly)
    assert 1.15 < np.median(r) < 1.35


def test_plummer_virial_ratio():
    pos, vel, m = gen.plummer(4096, 5)
    ke = 0.5 * (m * (vel ** 2).sum(1)).sum()
    d = pos[:, None, :] - pos[None]
    r = np.sqrt((d ** 2).sum(-1))
    np.fill_diagonal(r, np.inf)
    pe = -0.5 * (m[:, None] * m[None] / r).sum()
    assert 0.4 < 2 * ke / -pe < 1.6


def test_lognormal_masses_renormalised():
    _, _, m = gen.plummer(10000, 1002, masses="lognormal")
    assert abs(m.sum() - 1.0) < 1e-12
    lm = np.log(m * len(m))
    assert 0.4 < lm.std() < 0.6


def test_disk_shape():
    pos, vel, m = gen.exponential_disk(20000, 1003)
    assert abs(m[0] - 0.1) < 1e-15 and abs(m[1:].sum() - 1.0) < 1e-9
    R = np.hypot(pos[1:, 0], pos[1:, 1])
    assert R.max() <= 5.05  # truncation at 5 Rd, then COM centring
    assert abs(np.median(np.abs(pos[1:, 2])) - 0.1 * np.arctanh(0.5)) < 0.01
    vt = (pos[1:, 0] * vel[1:, 1] - pos[1:, 1] * vel[1:, 0]) / R
    assert (vt > 0).mean() > 0.99   # cold, rotating


def test_ensemble_layout():
    pos, vel, m, off = gen.hierarchical_ensemble(256, 1004)
    sizes = np.diff(off)
    assert sizes.min() >= 3 and sizes.max() <= 64
    assert off[-1] == len(m) == len(pos)
    for s in range(0, 256, 37):
        a, b = off[s], off[s + 1]
        M = m[a:b].sum()
        np.testing.assert_allclose((m[a:b, None] * pos[a:b]).sum(0) / M, 0, atol=1e-12)
        sep = np.linalg.norm(pos[a] - pos[a + 1])
        assert sep <= 0.1 * 1.9 + 1e-12
