"""ElasticityModule parity against the CPU restatement.  The bonds come from
the same neighbour list on both sides (the restatement's, uploaded), so the
rest shapes must agree bit for bit; K^-1 within 1e-5 relative; positions
within 1e-5 relative after one solve and 1e-4 after 10 steps."""
import numpy as np
import pytest
import torch

import scenes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def t(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def setup(ctx, oracle, dims, cap, seed=0):
    sc = scenes.elastic_bar(seed=seed, dims=dims, cap=cap)
    # jitter the lattice slightly so capped lists have no distance ties
    rng = np.random.default_rng(seed)
    sc.x = (sc.x + rng.uniform(-0.02, 0.02, sc.x.shape) * sc.spacing).astype(np.float32)
    ri, re = oracle.neighbor_query(sc.x, sc.horizon, sc.lo, sc.hi, cap)
    total = re.shape[0]
    ctx_x = t(sc.x)
    ctx.pd_init(ctx_x, t(ri, np.int32), t(re, np.int32), cap, total, sc.horizon)
    ctx.pd_set_bulk(t(sc.bulk))
    return sc, ri, re, total


@pytest.mark.parametrize("cap", [80, 0])
def test_rest_shape_and_inverse_k(ctx, oracle, cap):
    sc, ri, re, total = setup(ctx, oracle, (16, 8, 8), cap)
    n = sc.x.shape[0]
    bonds = n * cap if cap else total
    gidx = torch.empty(bonds, dtype=torch.int32, device="cuda")
    gpos = torch.empty(3 * bonds, dtype=torch.float32, device="cuda")
    ginv = torch.empty(9 * n, dtype=torch.float32, device="cuda")
    ctx.pd_get_rest_shape(gidx, gpos, ginv)
    oidx, opos = oracle.pd_rest_shape(sc.x, ri, re, cap)
    oinv = oracle.pd_inverse_k(ri, cap, total, opos, sc.horizon)
    cnt = ri if cap else np.diff(np.r_[ri, total])
    valid = np.zeros(bonds, bool)
    for i in range(n):
        s = i * cap if cap else ri[i]
        valid[s:s + cnt[i]] = True
    assert np.array_equal(gidx.cpu().numpy()[valid], oidx[valid])
    assert np.array_equal(gpos.cpu().numpy().reshape(-1, 3)[valid], opos.reshape(-1, 3)[valid])
    assert rel(ginv.cpu().numpy(), oinv.reshape(-1)) < 1e-5


@pytest.mark.parametrize("cap", [80, 0])
def test_pd_steps(ctx, oracle, cap):
    sc, ri, re, total = setup(ctx, oracle, (16, 8, 8), cap, seed=1)
    v0 = np.random.default_rng(1).normal(0, 0.05, sc.x.shape).astype(np.float32)
    x, v = t(sc.x), t(v0)
    oidx, opos = oracle.pd_rest_shape(sc.x, ri, re, cap)
    oinv = oracle.pd_inverse_k(ri, cap, total, opos, sc.horizon)
    xo, vo = sc.x.copy(), v0.copy()
    for step in range(10):
        ctx.integrate(x, v, (0, -9.8, 0), sc.dt)
        ctx.pd_solve(x, v, sc.horizon, sc.mu, sc.lam, sc.iterations, sc.dt)
        xo, vo = oracle.integrate(xo, vo, (0, -9.8, 0), sc.dt)
        xo, vo = oracle.pd_solve(xo, vo, ri, cap, total, oidx, opos, oinv, sc.bulk, sc.horizon,
                                 sc.mu, sc.lam, sc.iterations, sc.dt)
        if step in (0, 9):
            ctx.check_status()
            tol = 1e-5 if step == 0 else 1e-4
            assert rel(x.cpu().numpy(), xo) < tol, step
