"""Size-independent properties at the benchmark's full size (2,097,152
particles, cap 64), beside the entry-by-entry comparisons with the CPU
restatement at that size (test_gpu_parity_at_size.py): the dynamic list is
symmetric; every capped row is the cap-nearest subset of the dynamic row
(count min(cap, |row|), every kept distance <= every dropped one up to float
rounding); the Jacobi solve conserves momentum (each pair's displacement
enters both ends with opposite signs); and, on a 16^3 block, the float fused
frame against a double run of the same method."""
import numpy as np
import pytest
import torch

import pkhot
import scenes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def big():
    sc = scenes.dam_break_2m(seed=0)
    return sc, torch.from_numpy(sc.x).cuda()


def test_lists_at_2m(ctx, big):
    sc, x = big
    n = x.shape[0]
    di, de, dtot = ctx.nq_build(x, sc.radius, sc.lo, sc.hi, 0)
    dcnt = torch.diff(torch.cat([di.long(), torch.tensor([dtot], device="cuda")]))
    src = torch.repeat_interleave(torch.arange(n, device="cuda"), dcnt)
    dst = de.long()
    fwd = torch.sort(src * n + dst).values
    bwd = torch.sort(dst * n + src).values
    assert torch.equal(fwd, bwd), "dynamic list not symmetric"
    ci, ce, _ = ctx.nq_build(x, sc.radius, sc.lo, sc.hi, sc.cap)
    ccnt = ci.long()
    assert torch.equal(ccnt, torch.clamp(dcnt, max=sc.cap)), "capped counts differ from min(cap, |row|)"
    ce = ce.view(n, sc.cap).long()
    slot = torch.arange(sc.cap, device="cuda").unsqueeze(0) < ccnt.unsqueeze(1)
    csrc = torch.arange(n, device="cuda").unsqueeze(1).expand(n, sc.cap)[slot]
    cdst = ce[slot]
    ckey = csrc * n + cdst
    pos = torch.searchsorted(fwd, ckey)
    assert torch.equal(fwd[pos.clamp(max=fwd.numel() - 1)], ckey), "capped entry missing from the dynamic row"
    # kept distances never exceed dropped ones
    xd = x.double()
    d2 = lambda a, b: ((xd[a] - xd[b]) ** 2).sum(1)
    kept = torch.full((n,), -1.0, dtype=torch.float64, device="cuda").scatter_reduce(
        0, csrc, d2(csrc, cdst), reduce="amax")
    in_cap = torch.zeros(fwd.numel(), dtype=torch.bool, device="cuda")
    in_cap[pos] = True
    fsrc, fdst = fwd // n, fwd % n
    drop = ~in_cap
    dropped = torch.full((n,), float("inf"), dtype=torch.float64, device="cuda").scatter_reduce(
        0, fsrc[drop], d2(fsrc[drop], fdst[drop]), reduce="amin")
    bad = kept > dropped * (1.0 + 1e-6)
    assert int(bad.sum()) == 0, f"{int(bad.sum())} rows keep a farther neighbour than one they drop"
    assert int(drop.sum()) > 0  # the cap does cut rows at this density


def test_solve_conserves_momentum_at_2m(ctx, big):
    sc, x0 = big
    x = x0.clone()
    v = torch.zeros_like(x)
    ctx.nq_build(x, sc.radius, sc.lo, sc.hi, sc.cap, want_list=False)
    ctx.integrate(x, v, sc.gravity, sc.dt)
    before = x.double().clone()
    prm = pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt)
    ctx.pbd_solve(x, v, None, None, sc.cap, 0, prm)
    ctx.check_status()
    dx = x.double() - before
    moved = float(dx.abs().sum())
    assert moved > 0.0
    assert float(dx.sum(0).abs().max()) < 1e-5 * moved


def test_float_frames_against_double_run(ctx, oracle):
    # away from the walls (no boundary contact in 10 frames): the float fused
    # frame against a double run of the same method (lists from the double
    # positions rounded to float, double integration and Jacobi solve)
    sc = scenes.dam_break_small(seed=8, n_side=16)
    x0 = (sc.x + np.array([0.3, 0.4, 0.3], np.float32)).astype(np.float32)
    v0 = np.random.default_rng(8).normal(0, 0.05, x0.shape).astype(np.float32)
    x, v = torch.from_numpy(x0).cuda(), torch.from_numpy(v0).cuda()
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt),
                           sc.gravity, boundary=False)
    f, m = oracle.density_scaling(sc.spacing, sc.radius, sc.rest_density)
    xo, vo = x0.astype(np.float64), v0.astype(np.float64)
    for step in range(10):
        ctx.pbf_step(x, v, prm)
        ri, re = oracle.neighbor_query(xo.astype(np.float32), sc.radius, sc.lo, sc.hi, sc.cap)
        xo, vo = oracle.integrate(xo, vo, sc.gravity, sc.dt, dtype=np.float64)
        xo, vo, _ = oracle.pbd_constrain(xo, vo, ri, re, sc.cap, sc.radius, f * m, sc.iterations, sc.dt,
                                         dtype=np.float64)
        if step in (0, 9):
            ctx.check_status()
            assert rel(x.cpu().numpy(), xo) < 1e-4, step
