"""The N-body Einstein-Infeld-Hoffmann 1PN acceleration of the oracle (the
FP64 CPU checker for the ensemble kernel's EIH force law), pinned three ways
with no GPU:

1. Two unsoftened bodies: EIH equals the reference's pairwise get_pn1
   (tool_chain_impl.cpp:110-137, through the oracle's pair law, itself pinned
   to the reference's own outputs in test_oracle.py) to 1e-14.
2. The published EIH Lagrangian (Landau & Lifshitz, The Classical Theory of
   Fields, sec. 106; Poisson & Will, Gravity, 2014, sec. 9.3): its
   Euler-Lagrange accelerations, computed here by automatic differentiation
   of the Lagrangian (torch, FP64), agree with the oracle's EIH accelerations
   up to terms of order c^-4, so the mismatch falls 16x per doubling of c
   (asserted >= 12x). The pairwise law, which drops the three-body terms,
   misses by order c^-2 (4x per doubling; asserted <= 6x), so the check has
   teeth.
3. The conserved energy of that Lagrangian (E = v.dL/dv - L, the oracle's
   EIH energy) drifts along an EIH trajectory by an amount that falls as
   c^-4 (the truncation of the 1PN equations), and along the pairwise one by
   a c^-2 amount, far larger.
"""
import numpy as np
import pytest

from oracle.oracle import EIH, NEWTON, PN1


def _lagrangian(x, v, m, G, c):
    """L = sum_a m_a v_a^2 / 2 + 1/2 sum_{a != b} G m_a m_b / r_ab
         + c^-2 [ sum_a m_a v_a^4 / 8
                  + 1/2 sum_{a != b} (G m_a m_b / r_ab) (3/2 (v_a^2 + v_b^2) - 7/2 v_a.v_b
                                                        - 1/2 (n_ab.v_a)(n_ab.v_b))
                  - 1/2 sum_a m_a phi_a^2 ],   phi_a = sum_{b != a} G m_b / r_ab"""
    import torch
    n = len(m)
    d = x[:, None, :] - x[None, :, :]
    eye = torch.eye(n, dtype=torch.bool)
    r = torch.sqrt((d * d).sum(-1) + eye.double())
    inv = torch.where(eye, torch.zeros_like(r), 1.0 / r)
    nab = d * inv[..., None]
    v2 = (v * v).sum(-1)
    mm = m[:, None] * m[None, :]
    nva = (nab * v[:, None, :]).sum(-1)
    nvb = (nab * v[None, :, :]).sum(-1)
    X = 1.5 * (v2[:, None] + v2[None, :]) - 3.5 * (v @ v.T) - 0.5 * nva * nvb
    phi = (G * m[None, :] * inv).sum(1)
    L0 = 0.5 * (m * v2).sum() + 0.5 * (G * mm * inv).sum()
    L1 = (m * v2 * v2).sum() / 8 + 0.5 * (G * mm * inv * X).sum() - 0.5 * (m * phi * phi).sum()
    return L0 + L1 / c ** 2


def _euler_lagrange_acc(x, v, m, G, c):
    """Solve d/dt dL/dv = dL/dx for the accelerations:
    (d2L/dv2) a = dL/dx - (d2L/dv dx) v."""
    import torch
    n = len(m)
    xt, vt, mt = (torch.tensor(np.asarray(a, dtype=np.float64)) for a in (x, v, m))
    xf, vf = xt.reshape(-1), vt.reshape(-1)

    def f(xa, va):
        return _lagrangian(xa.reshape(n, 3), va.reshape(n, 3), mt, G, c)

    H = torch.autograd.functional.hessian(f, (xf, vf))
    xg = xf.clone().requires_grad_()
    gx = torch.autograd.grad(f(xg, vf), xg)[0]
    a = torch.linalg.solve(H[1][1], gx - H[1][0] @ vf)
    return a.reshape(n, 3).numpy()


def _pairwise(orc, x, v, m, G, c):
    n = len(m)
    return np.array([sum(orc.pair_acc(G, 1.0 / c, 0.0, NEWTON | PN1, m[i], m[j], v[i], v[j], x[i], x[j])
                         for j in range(n) if j != i) for i in range(n)])


def test_two_bodies_reduce_to_reference_pairwise_law(orc):
    rng = np.random.default_rng(31)
    for _ in range(8):
        x, v, m = rng.normal(size=(2, 3)), rng.normal(size=(2, 3)), rng.uniform(0.1, 2.0, 2)
        for c in (3.0, 30.0):
            a = orc.eih_acc(x, v, m, 1.0, c)
            ref = _pairwise(orc, x, v, m, 1.0, c)
            assert np.abs(a - ref).max() < 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("n,seed", [(3, 32), (5, 33), (12, 34)])
def test_eih_is_the_euler_lagrange_flow_of_the_eih_lagrangian(orc, n, seed):
    pytest.importorskip("torch")
    rng = np.random.default_rng(seed)
    x, v, m = rng.normal(size=(n, 3)), 0.5 * rng.normal(size=(n, 3)), rng.uniform(0.5, 1.5, n)
    cs = (20.0, 40.0, 80.0)
    eih, pw = [], []
    for c in cs:
        el = _euler_lagrange_acc(x, v, m, 1.0, c)
        eih.append(np.linalg.norm(orc.eih_acc(x, v, m, 1.0, c) - el))
        pw.append(np.linalg.norm(_pairwise(orc, x, v, m, 1.0, c) - el))
    for k in range(len(cs) - 1):
        assert eih[k] / eih[k + 1] >= 12.0, eih   # O(c^-4): 16x per doubling
        assert pw[k] / pw[k + 1] <= 6.0, pw       # O(c^-2): 4x per doubling
    pn_part = np.linalg.norm(orc.eih_acc(x, v, m, 1.0, cs[-1]) - orc.eih_acc(x, v, m, 1.0, 1e30))
    assert eih[-1] < 0.05 * pn_part


def test_eih_energy_is_the_lagrangian_energy(orc):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(36)
    n = 7
    x, v, m = rng.normal(size=(n, 3)), 0.5 * rng.normal(size=(n, 3)), rng.uniform(0.5, 1.5, n)
    xt, vt, mt = (torch.tensor(a) for a in (x, v, m))
    vt.requires_grad_()
    L = _lagrangian(xt, vt, mt, 1.0, 20.0)
    g = torch.autograd.grad(L, vt)[0]
    e = float(((g * vt).sum() - L).detach())
    assert abs(orc.ens_energy(np.array([0, n]), x, v, m, c=20.0, pn=NEWTON | PN1 | EIH)[0] - e) < 1e-14 * abs(e)


def test_eih_trajectory_keeps_the_eih_energy(orc):
    """A compact 6-body system (v ~ 0.5, unsoftened), 4000 Yoshida-4 steps of
    dt = 1e-4 at c = 20 and 40: the EIH energy drifts less than 0.1x as much (measured
    0.04x) along the EIH flow as along the pairwise flow, and that drift falls
    as c^-4 (measured 17x from c = 20 to 40; asserted >= 10x), the pairwise
    one as c^-2 (4x; asserted <= 6x). The step is small enough that the
    integration error is far below both."""
    rng = np.random.default_rng(35)
    n = 6
    x, v, m = rng.normal(size=(n, 3)), 0.5 * rng.normal(size=(n, 3)), rng.uniform(0.5, 1.5, n)
    off = np.array([0, n])
    dt, steps = 1e-4, 4000
    drift = {}
    for c in (20.0, 40.0):
        e0 = orc.ens_energy(off, x, v, m, c=c, pn=NEWTON | PN1 | EIH)[0]
        for name, law in (("eih", NEWTON | PN1 | EIH), ("pairwise", NEWTON | PN1)):
            p, u = orc.ens_run(off, x, v, m, dt, steps, c=c, integrator=1, pn=law)
            drift[name, c] = abs(orc.ens_energy(off, p, u, m, c=c, pn=NEWTON | PN1 | EIH)[0] - e0) / abs(e0)
    assert drift["eih", 20.0] < 0.1 * drift["pairwise", 20.0], drift
    assert drift["eih", 20.0] / drift["eih", 40.0] >= 10.0, drift
    assert drift["pairwise", 20.0] / drift["pairwise", 40.0] <= 6.0, drift
