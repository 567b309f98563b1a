"""Differentiable peridynamics rollouts: the rollout equals step-by-step
integrate + pk_pd_solve bit for bit; float and double rollouts agree; the
hand-written adjoint matches central finite differences of double rollouts
(eps 1e-4, relative 1e-3) and the float adjoint matches the double one; a few
gradient steps recover stiffness and initial velocity toward a target."""
import numpy as np
import pytest
import torch

import pkhot
import scenes
from pk_torch import RolloutSettings, pd_rollout

pytestmark = pytest.mark.gpu

DIMS = (8, 6, 6)


def t(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def block(ctx, oracle, seed=0, cap=80):
    sc = scenes.elastic_bar(seed=seed, dims=DIMS, cap=cap, stiffness=(0.5e4, 2.0e4))
    rng = np.random.default_rng(seed)
    sc.x = (sc.x + rng.uniform(-0.02, 0.02, sc.x.shape) * sc.spacing).astype(np.float32)
    ri, re = oracle.neighbor_query(sc.x, sc.horizon, sc.lo, sc.hi, cap)
    ctx.pd_init(t(sc.x), t(ri, np.int32), t(re, np.int32), cap, re.shape[0], sc.horizon)
    return sc


def test_rollout_equals_module_steps(ctx, oracle):
    sc = block(ctx, oracle)
    v0 = np.random.default_rng(1).normal(0, 0.05, sc.x.shape).astype(np.float32)
    ctx.pd_set_bulk(t(sc.bulk))
    x1, v1 = t(sc.x), t(v0)
    ctx.pd_rollout(x1, v1, sc.horizon, sc.mu, sc.lam, sc.iterations, sc.dt, steps=12, checkpoint_every=5)
    x2, v2 = t(sc.x), t(v0)
    for _ in range(12):
        ctx.integrate(x2, v2, (0.0, -9.8, 0.0), sc.dt)
        ctx.pd_solve(x2, v2, sc.horizon, sc.mu, sc.lam, sc.iterations, sc.dt)
    ctx.check_status()
    assert torch.equal(x1, x2) and torch.equal(v1, v2)


def test_float_and_double_rollouts_agree(ctx, oracle):
    sc = block(ctx, oracle, seed=2)
    v0 = np.random.default_rng(2).normal(0, 0.05, sc.x.shape)
    ctx.pd_set_bulk(t(sc.bulk))
    xf, vf = t(sc.x), t(v0)
    ctx.pd_rollout(xf, vf, sc.horizon, sc.mu, sc.lam, sc.iterations, sc.dt, steps=10)
    xd, vd = t(sc.x, np.float64), t(v0, np.float64)
    ctx.pd_rollout(xd, vd, sc.horizon, sc.mu, sc.lam, sc.iterations, sc.dt, steps=10,
                   bulk64=t(sc.bulk, np.float64))
    ctx.check_status()
    # FP32 against the FP64 run of the same method after 10 steps
    d = (xf.double() - xd).norm() / xd.norm()
    assert float(d) < 1e-4


def loss_fn(x, target):
    return ((x - target) ** 2).sum(dim=1).mean()


def test_adjoint_matches_finite_differences(ctx, oracle):
    sc = block(ctx, oracle, seed=3)
    n = sc.x.shape[0]
    s = RolloutSettings(horizon=sc.horizon, mu=sc.mu, lam=sc.lam, iterations=sc.iterations, dt=sc.dt,
                        steps=20, checkpoint_every=5)
    rng = np.random.default_rng(3)
    # target from hidden stiffness and initial velocity
    bulk_true = rng.uniform(0.5e4, 2.0e4, n)
    v_true = rng.normal(0, 0.05, (n, 3))
    x0 = t(sc.x, np.float64)
    with torch.no_grad():
        target = pd_rollout(x0, t(v_true, np.float64), t(bulk_true, np.float64), ctx, s)
    bulk = t(np.full(n, 1.0e4), np.float64).requires_grad_(True)
    v0 = t(rng.normal(0, 0.05, (n, 3)), np.float64).requires_grad_(True)
    loss = loss_fn(pd_rollout(x0, v0, bulk, ctx, s), target)
    loss.backward()
    gb, gv = bulk.grad.cpu().numpy(), v0.grad.cpu().numpy()

    def dL(bp, vp, bm, vm):
        # L(+) - L(-) from the two trajectories (no cancellation of two losses)
        with torch.no_grad():
            xp, xm = pd_rollout(x0, vp, bp, ctx, s), pd_rollout(x0, vm, bm, ctx, s)
            return float(((xp - xm) * (xp + xm - 2.0 * target)).sum(dim=1).mean())

    pick = np.random.default_rng(4)
    bad = []
    for k in pick.choice(n, 16, replace=False):
        eps = 1e-4 * 1.0e4
        bp, bm = bulk.detach().clone(), bulk.detach().clone()
        bp[k] += eps
        bm[k] -= eps
        fd = dL(bp, v0.detach(), bm, v0.detach()) / (2 * eps)
        if abs(fd - gb[k]) > 1e-3 * max(abs(fd), 1e-3 * np.abs(gb).max()):
            bad.append(("bulk", int(k), fd, gb[k]))
    for k in pick.choice(n * 3, 16, replace=False):
        eps = 1e-4
        vp, vm = v0.detach().clone(), v0.detach().clone()
        vp.view(-1)[k] += eps
        vm.view(-1)[k] -= eps
        fd = dL(bulk.detach(), vp, bulk.detach(), vm) / (2 * eps)
        g = gv.reshape(-1)[k]
        if abs(fd - g) > 1e-3 * max(abs(fd), 1e-3 * np.abs(gv).max()):
            bad.append(("v0", int(k), fd, g))
    assert not bad, bad[:5]

    # the float adjoint against the double one, same seed dL/dx_T
    seed = t(np.random.default_rng(6).normal(0, 1, (n, 3)), np.float64)
    vv = v0.detach()
    xd, vd = x0.clone(), vv.clone()
    ctx.pd_rollout(xd, vd, s.horizon, s.mu, s.lam, s.iterations, s.dt, s.steps, s.checkpoint_every,
                   bulk64=bulk.detach())
    gx64, gv64, gb64 = ctx.pd_rollout_backward(seed)
    ctx.pd_set_bulk(bulk.detach().float())
    xf, vf = x0.float(), vv.float()
    ctx.pd_rollout(xf, vf, s.horizon, s.mu, s.lam, s.iterations, s.dt, s.steps, s.checkpoint_every)
    gx32, gv32, gb32 = ctx.pd_rollout_backward(seed.float())
    ctx.check_status()
    for a, b in ((gx32, gx64), (gv32, gv64), (gb32, gb64)):
        r = float((a.double() - b).norm() / b.norm())
        assert r < 1e-3, r


def test_gradient_descent_recovers_parameters(ctx, oracle):
    sc = block(ctx, oracle, seed=5)
    n = sc.x.shape[0]
    s = RolloutSettings(horizon=sc.horizon, mu=sc.mu, lam=sc.lam, iterations=sc.iterations, dt=sc.dt,
                        steps=20, checkpoint_every=10)
    rng = np.random.default_rng(5)
    x0 = t(sc.x, np.float64)
    with torch.no_grad():
        target = pd_rollout(x0, t(rng.normal(0, 0.05, (n, 3)), np.float64),
                            t(rng.uniform(0.5e4, 2.0e4, n), np.float64), ctx, s)
    log_b = torch.full((n,), float(np.log(1.0e4)), dtype=torch.float64, device="cuda", requires_grad=True)
    v0 = torch.zeros((n, 3), dtype=torch.float64, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([{"params": [log_b], "lr": 0.05}, {"params": [v0], "lr": 0.01}])
    losses = []
    for _ in range(30):
        opt.zero_grad()
        loss = loss_fn(pd_rollout(x0, v0, torch.exp(log_b), ctx, s), target)
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
    assert losses[-1] < 0.05 * losses[0], losses[::5]
