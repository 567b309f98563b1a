"""FixedPoints (pins and the plane constraint) and the peridynamics bar of the
benchmark configuration (left end clamped, right end pulled, bonds breaking at
2% stretch) against the CPU restatement."""
import numpy as np
import pytest
import torch

import pkhot
import scenes

pytestmark = pytest.mark.gpu


def t(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_pins_and_plane_bit_exact(ctx, oracle):
    rng = np.random.default_rng(3)
    n = 5000
    x0 = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    v0 = rng.normal(0, 1, (n, 3)).astype(np.float32)
    ids = rng.choice(n, 300, replace=False).astype(np.int32)
    tgt = rng.uniform(-1, 1, (300, 3)).astype(np.float32)
    vel = rng.normal(0, 1, (300, 3)).astype(np.float32)
    for with_vel in (False, True):
        x, v = t(x0), t(v0)
        ctx.fixed_points(x, v, t(ids, np.int32), t(tgt), t(vel) if with_vel else None)
        xo, vo = oracle.fixed_points(x0, v0, ids, tgt, vel if with_vel else None)
        ctx.check_status()
        assert np.array_equal(x.cpu().numpy(), xo) and np.array_equal(v.cpu().numpy(), vo)
    d = np.array([0.3, -0.5, 0.81], np.float32)
    d = (d / np.linalg.norm(d)).astype(np.float32)
    x = t(x0)
    ctx.plane_constrain(x, (0.1, 0.2, -0.1), d)
    xo = oracle.plane_constrain(x0, (0.1, 0.2, -0.1), d)
    assert np.array_equal(x.cpu().numpy(), xo)


def test_pin_with_bad_id_is_reported(ctx):
    x = t(np.zeros((10, 3)))
    v = t(np.zeros((10, 3)))
    ctx.fixed_points(x, v, t(np.array([2, 10], np.int32), np.int32), t(np.ones((2, 3))))
    assert ctx.status() == pkhot.PK_ERR_ARG
    assert np.all(x.cpu().numpy()[2] == 1.0)  # the valid pin was applied
    assert ctx.status() == pkhot.PK_OK


def test_pulled_bar_with_bond_break(ctx, oracle):
    # the benchmark's elastic bar on a smaller lattice: x-index 0 clamped,
    # the last x layer pulled at 0.5 m/s, bonds break beyond 2% stretch.  The
    # pulled layer moves 1/8 spacing per step, so bonds at that end tear from
    # the first step on and the motion becomes chaotic (float and double runs
    # of the restatement part within a few dozen steps): compare 3 steps.
    dims = (24, 6, 6)
    sc = scenes.elastic_bar(seed=2, dims=dims, cap=80)
    rng = np.random.default_rng(2)
    sc.x = (sc.x + rng.uniform(-0.02, 0.02, sc.x.shape) * sc.spacing).astype(np.float32)
    n = sc.x.shape[0]
    ix = np.arange(n) // (dims[1] * dims[2])
    left = np.nonzero(ix == 0)[0].astype(np.int32)
    right = np.nonzero(ix == dims[0] - 1)[0].astype(np.int32)
    pull = np.array([0.5, 0.0, 0.0], np.float32)
    ri, re = oracle.neighbor_query(sc.x, sc.horizon, sc.lo, sc.hi, sc.cap)
    total = re.shape[0]
    x, v = t(sc.x), t(sc.v)
    ctx.pd_init(x, t(ri, np.int32), t(re, np.int32), sc.cap, total, sc.horizon)
    ctx.pd_set_bulk(t(sc.bulk))
    oidx, opos = oracle.pd_rest_shape(sc.x, ri, re, sc.cap)
    oinv = oracle.pd_inverse_k(ri, sc.cap, total, opos, sc.horizon)
    alive = np.ones(n * sc.cap, np.uint8)
    ids = np.concatenate([left, right])
    vel = np.zeros((ids.shape[0], 3), np.float32)
    vel[left.shape[0]:] = pull
    dt = np.float32(sc.dt)
    xo, vo = sc.x.copy(), sc.v.copy()
    steps = 3
    for step in range(steps):
        tgt = sc.x[ids].copy()
        tgt[left.shape[0]:] += np.float32(step + 1) * dt * pull  # the pulled end's target
        tgt = tgt.astype(np.float32)
        ids_t, tgt_t, vel_t = t(ids, np.int32), t(tgt), t(vel)
        ctx.integrate(x, v, (0, 0, 0), sc.dt)
        ctx.fixed_points(x, v, ids_t, tgt_t, vel_t)
        ctx.pd_solve(x, v, sc.horizon, sc.mu, sc.lam, sc.iterations, sc.dt, sc.break_stretch)
        ctx.fixed_points(x, v, ids_t, tgt_t, vel_t)
        xo, vo = oracle.integrate(xo, vo, (0, 0, 0), sc.dt)
        xo, vo = oracle.fixed_points(xo, vo, ids, tgt, vel)
        oracle.pd_break(xo, ri, sc.cap, total, oidx, opos, alive, sc.break_stretch)
        xo, vo = oracle.pd_solve(xo, vo, ri, sc.cap, total, oidx, opos, oinv, sc.bulk, sc.horizon,
                                 sc.mu, sc.lam, sc.iterations, sc.dt, alive=alive)
        xo, vo = oracle.fixed_points(xo, vo, ids, tgt, vel)
    ctx.check_status()
    xg = x.cpu().numpy()
    assert rel(xg, xo) < 1e-4
    # the pulled end moved by steps * dt * 0.5 m/s and bonds near it broke
    assert np.allclose(xg[right, 0] - sc.x[right, 0], steps * sc.dt * 0.5, atol=1e-6)
    assert alive.sum() < n * sc.cap  # something broke at 2% stretch
