"""Hand-written leapfrog adjoint against the FP64 CPU reverse-mode reference
(oracle/aster_oracle.c, orc_adjoint) and central finite differences.

Tolerances (relative L2 over the gradient arrays): FP64 adjoint vs CPU
reverse mode 1e-10; mixed (FP32 forces and adjoint pair terms, FP64 state)
1e-5. C5 at full size (N = 16384 Plummer, eps = 0.01, dt = 1e-3, 1000 steps,
checkpoints every 32): mixed adjoint vs central differences (h = 1e-6, FP64
forward) on 64 random coordinates of x0 and v0, relative L2 < 1e-4.
"""
import numpy as np
import pytest

from aster_b200 import gen
from aster_b200.api import FP64, MIXED, SOLVER_ALLPAIRS, Params
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _setup(n, T, dt, eps2, seed):
    x0, v0, m = gen.plummer(n, seed)
    return x0, v0, m


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-10), (MIXED, 1e-5)])
def test_adjoint_vs_cpu_reverse_mode(ctx, orc, prec, tol):
    n, T, dt, eps2 = 256, 60, 1e-3, 1e-4
    x0, v0, m = gen.plummer(n, 3)
    target, _, _, _ = orc.kdk(x0 + np.random.default_rng(2).normal(0, 1e-3, x0.shape), v0, m, dt, T, eps2=eps2)
    loss_c, gx_c, gv_c, gm_c = orc.adjoint(x0, v0, m, target, dt, T, eps2=eps2)
    ctx.upload(x0, v0, m)
    loss, gx, gv, gm = ctx.adjoint(Params(eps2=eps2, dt=dt), T, target, prec, checkpoint_every=7)
    assert abs(loss - loss_c) < tol * abs(loss_c)
    assert rel_l2(gx, gx_c) < tol
    assert rel_l2(gv, gv_c) < tol
    assert rel_l2(gm, gm_c) < tol
    # the uploaded state is left unchanged
    p0, vv0, _ = ctx.download()
    np.testing.assert_array_equal(p0, x0)
    np.testing.assert_array_equal(vv0, v0)


def test_checkpoint_interval_does_not_change_the_result(ctx, orc):
    n, T, dt, eps2 = 300, 45, 1e-3, 1e-4
    x0, v0, m = gen.plummer(n, 8)
    target = x0 + 1e-3
    ctx.upload(x0, v0, m)
    ref = ctx.adjoint(Params(eps2=eps2, dt=dt), T, target, FP64, checkpoint_every=1)
    for K in (4, 32, 45, 100):
        got = ctx.adjoint(Params(eps2=eps2, dt=dt), T, target, FP64, checkpoint_every=K)
        for a, b in zip(ref[1:], got[1:]):
            np.testing.assert_array_equal(a, b)  # recomputation reproduces the forward pass bit for bit


def test_torch_autograd_wrapper(ctx):
    torch = pytest.importorskip("torch")
    from aster_b200.autograd import leapfrog_loss
    n, T, dt, eps2 = 200, 30, 1e-3, 1e-4
    x0, v0, m = gen.plummer(n, 4)
    target = x0 + 2e-3
    p = Params(eps2=eps2, dt=dt)
    X = torch.tensor(x0, requires_grad=True)
    V = torch.tensor(v0, requires_grad=True)
    M = torch.tensor(m, requires_grad=True)
    loss = leapfrog_loss(X, V, M, torch.tensor(target), p, T, FP64, 16, ctx)
    (2.0 * loss).backward()
    ctx.upload(x0, v0, m)
    l2, gx, gv, gm = ctx.adjoint(p, T, target, FP64, 16)
    assert abs(loss.item() - l2) < 1e-15 * max(1.0, abs(l2))
    np.testing.assert_allclose(X.grad.numpy(), 2 * gx, rtol=1e-14, atol=0)
    np.testing.assert_allclose(V.grad.numpy(), 2 * gv, rtol=1e-14, atol=0)
    np.testing.assert_allclose(M.grad.numpy(), 2 * gm, rtol=1e-14, atol=0)


def _fd_loss(ctx, x0, v0, m, p, T, target):
    ctx.upload(x0, v0, m)
    ctx.kdk_steps(p, T, SOLVER_ALLPAIRS, FP64)
    xT, _, _ = ctx.download()
    return float(((xT - target) ** 2).sum() / len(m))


def test_c5_full_size_vs_finite_differences(ctx):
    n, T, dt, eps = 16384, 1000, 1e-3, 0.01
    p = Params(eps2=eps * eps, dt=dt)
    x0, v0, m = gen.plummer(n, 1005)
    rng = np.random.default_rng(1005)
    ctx.upload(x0 + rng.normal(0, 1e-3, x0.shape), v0, m)
    ctx.kdk_steps(p, T, SOLVER_ALLPAIRS, FP64)
    target, _, _ = ctx.download()
    ctx.upload(x0, v0, m)
    loss, gx, gv, gm = ctx.adjoint(p, T, target, MIXED, checkpoint_every=32)
    h = 1e-6
    pick = rng.choice(2 * n * 3, 64, replace=False)
    g_ad, g_fd = [], []
    for f in pick:
        which, flat = divmod(int(f), n * 3)
        i, a = divmod(flat, 3)
        base = [x0.copy(), v0.copy()]
        plus = [b.copy() for b in base]
        minus = [b.copy() for b in base]
        plus[which][i, a] += h
        minus[which][i, a] -= h
        fd = (_fd_loss(ctx, plus[0], plus[1], m, p, T, target) - _fd_loss(ctx, minus[0], minus[1], m, p, T, target)) / (2 * h)
        g_fd.append(fd)
        g_ad.append((gx if which == 0 else gv)[i, a])
    g_ad, g_fd = np.array(g_ad), np.array(g_fd)
    err = np.linalg.norm(g_ad - g_fd) / np.linalg.norm(g_fd)
    assert err < 1e-4, err
