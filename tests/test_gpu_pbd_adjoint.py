"""The differentiable DensityPBD rollout (pk_pbd_rollout / _backward and the
double-precision pair), on fluid blocks with the 32,768-particle dam break's
parameters, moved off the walls (the differentiable frame has no boundary),
initial velocities N(0, 0.05^2), 20 frames, checkpoints every 5.

- The float rollout is the fused frame (pk_pbf_step without boundary) bit for
  bit; the double rollout stays within 1e-5 of it after 20 frames.
- The double adjoint matches central finite differences of the double rollout
  (eps 1e-4 on the initial velocity, 1e-5 on the initial position) to 1e-3
  relative on 64 coordinates.  The frame map is smooth except where lambda's
  clamp switches (rho = 1000) or a capped row exchanges two members at equal
  distance; the check runs on dynamic lists (the spiky kernel and its first
  two derivatives vanish at the radius) on a block compressed to 0.9 spacing,
  and a coordinate counts as smooth where the differences at eps and 2 eps
  agree to 1e-4 (a clamp switch inside the stencil separates them).
  Coordinates are drawn (at most 96) until 64 smooth ones are found, and every
  one of the 64 must match.
- The float adjoint is within 2e-2 of the double one (the float and double
  trajectories differ by rounding, and the gradient of a map with clamp
  switches follows them).
- The autograd Function returns the adjoint.
- Gradient descent on the initial velocities recovers hidden ones (a smooth
  field: translation, rotation, shear) from the final positions: the
  velocity error falls below 5% of where it started.
"""
import numpy as np
import pytest
import torch

import pkhot
import pk_torch
import scenes

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def block(cap, seed=0, n_side=12, squeeze=1.0):
    sc = scenes.dam_break_small(seed=seed, n_side=n_side)
    c = sc.x.mean(axis=0)
    x0 = (c + (sc.x - c) * squeeze + np.array([0.4, 0.4, 0.4], np.float32)).astype(np.float32)
    v0 = np.random.default_rng(seed + 100).normal(0.0, 0.05, x0.shape).astype(np.float32)
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt),
                           sc.gravity, boundary=False)
    return sc, x0, v0, prm


def test_float_rollout_equals_fused_frames(ctx):
    sc, x0, v0, prm = block(60)
    xa, va = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(v0.copy()).cuda()
    xb, vb = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(v0.copy()).cuda()
    ctx.pbd_rollout(xa, va, prm, 20, 5)
    for _ in range(20):
        ctx.pbf_step(xb, vb, prm)
    ctx.check_status()
    assert torch.equal(xa, xb) and torch.equal(va, vb)


@pytest.mark.parametrize("cap", [60, 0])
def test_double_rollout_close_to_float(ctx, cap):
    sc, x0, v0, prm = block(cap)
    x32, v32 = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(v0.copy()).cuda()
    x64, v64 = x32.double(), v32.double()
    ctx.pbd_rollout(x32, v32, prm, 20, 5)
    ctx.pbd_rollout(x64, v64, prm, 20, 5)
    ctx.check_status()
    assert rel(x32.cpu().numpy(), x64.cpu().numpy()) < 1e-5
    assert rel(v32.cpu().numpy(), v64.cpu().numpy()) < 1e-3


def loss_and_grad(ctx, prm, x0, v0, target, steps=20, every=5):
    """L = mean_i |x_T,i - target_i|^2 and dL/dx0, dL/dv0 (the rollout's precision)."""
    x, v = x0.clone(), v0.clone()
    ctx.pbd_rollout(x, v, prm, steps, every)
    n = x.shape[0]
    L = float(((x - target) ** 2).sum()) / n
    gx, gv = ctx.pbd_rollout_backward(2.0 * (x - target) / n)
    return L, gx, gv, x


def fd_grad(ctx, prm, x0, v0, target, which, k, eps, steps=20, every=5):
    """Central difference of L in coordinate k of x0 or v0, from the
    trajectory difference: L(+) - L(-) = mean (x+ - x-) . (x+ + x- - 2 t)."""
    runs = []
    for sgn in (1.0, -1.0):
        x, v = x0.clone(), v0.clone()
        (x if which == "x" else v).view(-1)[k] += sgn * eps
        ctx.pbd_rollout(x, v, prm, steps, every)
        runs.append(x)
    xp, xm = runs
    dL = float(((xp - xm) * (xp + xm - 2.0 * target)).sum()) / xp.shape[0]
    return dL / (2.0 * eps)


def test_double_adjoint_matches_finite_differences(ctx):
    sc, x0, v0, prm = block(0, seed=3, n_side=16, squeeze=0.9)
    n = x0.shape[0]
    x0d, v0d = torch.from_numpy(x0).cuda().double(), torch.from_numpy(v0).cuda().double()
    # the target: a run from other initial velocities
    xt, vt = x0d.clone(), v0d.clone() * 0.5
    ctx.pbd_rollout(xt, vt, prm, 20, 5)
    target = xt
    L, gx, gv, _ = loss_and_grad(ctx, prm, x0d, v0d, target)
    ctx.check_status()
    assert L > 0.0
    rng = np.random.default_rng(7)
    # velocity and position coordinates (3 to 1), drawn until 64 smooth ones are found
    pool = rng.choice(3 * n, 96, replace=False)
    coords = [("x", int(k), 1e-5) if q % 4 == 3 else ("v", int(k), 1e-4) for q, k in enumerate(pool)]
    gvn, gxn = gv.view(-1).cpu().numpy(), gx.view(-1).cpu().numpy()
    scale = {"v": np.abs(gvn).max(), "x": np.abs(gxn).max()}
    errs, tried = [], 0
    for which, k, eps in coords:
        if len(errs) == 64:
            break
        tried += 1
        f1 = fd_grad(ctx, prm, x0d, v0d, target, which, k, eps)
        f2 = fd_grad(ctx, prm, x0d, v0d, target, which, k, 2.0 * eps)
        floor = 1e-3 * scale[which]
        if abs(f1 - f2) > 1e-4 * max(abs(f1), floor):
            continue  # a clamp switch inside the stencil
        adj = (gvn if which == "v" else gxn)[k]
        errs.append(abs(adj - f1) / max(abs(f1), floor))
    errs = np.array(errs)
    print(f"FD vs adjoint: {len(errs)} smooth of {tried} coordinates tried, max rel {errs.max():.2e}, "
          f"median {np.median(errs):.2e}")
    assert len(errs) == 64
    assert errs.max() < 1e-3


def test_float_adjoint_close_to_double(ctx):
    sc, x0, v0, prm = block(60, seed=4)
    xt, vt = torch.from_numpy(x0).cuda(), torch.from_numpy(v0).cuda() * 0.5
    ctx.pbd_rollout(xt, vt, prm, 20, 5)
    grads = {}
    for dt_ in (torch.float32, torch.float64):
        x0t = torch.from_numpy(x0).cuda().to(dt_)
        v0t = torch.from_numpy(v0).cuda().to(dt_)
        _, gx, gv, _ = loss_and_grad(ctx, prm, x0t, v0t, xt.to(dt_))
        grads[dt_] = (gx.double().cpu().numpy(), gv.double().cpu().numpy())
    ctx.check_status()
    assert rel(grads[torch.float32][1], grads[torch.float64][1]) < 2e-2
    assert rel(grads[torch.float32][0], grads[torch.float64][0]) < 2e-2


def test_autograd_function_gives_the_adjoint(ctx):
    sc, x0, v0, prm = block(60, seed=5)
    x0t = torch.from_numpy(x0).cuda().requires_grad_(True)
    v0t = torch.from_numpy(v0).cuda().requires_grad_(True)
    target = torch.from_numpy(x0).cuda()
    xT, vT = pk_torch.pbd_rollout(x0t, v0t, ctx, prm, 20, 5)
    loss = ((xT - target) ** 2).sum() / x0.shape[0] + (vT ** 2).sum() / x0.shape[0]
    loss.backward()
    x, v = torch.from_numpy(x0).cuda(), torch.from_numpy(v0).cuda()
    ctx.pbd_rollout(x, v, prm, 20, 5)
    gx, gv = ctx.pbd_rollout_backward(2.0 * (x - target) / x0.shape[0], 2.0 * v / x0.shape[0])
    assert torch.equal(x, xT.detach())
    assert torch.allclose(x0t.grad, gx) and torch.allclose(v0t.grad, gv)


def test_gradient_descent_recovers_initial_velocities(ctx):
    # hidden initial velocities: a smooth field (translation, rotation about the
    # block's centre and a volume-preserving shear), which the final positions
    # determine; the density constraint absorbs compressive components
    sc, x0, _, prm = block(60, seed=6)
    n = x0.shape[0]
    steps = 20
    c = x0.mean(axis=0)
    r = x0 - c
    omega = np.array([0.0, 0.0, 2.0])
    v_hidden = (np.array([0.03, -0.02, 0.01]) + np.cross(omega, r)
                + np.stack([1.5 * r[:, 1], np.zeros(n), np.zeros(n)], 1)).astype(np.float32)
    xt, vt = torch.from_numpy(x0).cuda(), torch.from_numpy(v_hidden).cuda()
    ctx.pbd_rollout(xt, vt, prm, steps, 5)
    target = xt
    x0t = torch.from_numpy(x0).cuda()
    vh = torch.from_numpy(v_hidden).cuda()
    v = torch.zeros_like(vh)  # the guess
    err0 = float(torch.linalg.norm(v - vh) / torch.linalg.norm(vh))
    # x_T moves by about steps*dt per unit of v0: step size of a Gauss-Newton-like descent
    eta = 0.5 * n / (2.0 * (steps * sc.dt) ** 2)
    for _ in range(30):
        _, _, gv, _ = loss_and_grad(ctx, prm, x0t, v, target, steps, 5)
        v = v - eta * gv
    ctx.check_status()
    err = float(torch.linalg.norm(v - vh) / torch.linalg.norm(vh))
    print(f"initial-velocity error: {err0:.3f} -> {err:.3f}")
    assert err < 0.05 * err0
