"""ImplicitViscosity parity against the CPU restatement (oracle
implicit_viscosity, ImplicitViscosity.cu:8-128): the generic-list entry point
on fixed and dynamic lists, and the fused frame's viscosity stage on the
solver rows.  Tolerance: velocities within 1e-5 relative (2-norm) for the
sweeps alone; the fused frame keeps the DensityPBD bounds (1e-4 positions,
1e-3 velocities after 10 frames).  Sums run in list order on both sides, so
the differences are FP32 rounding of the weights only."""
import numpy as np
import pytest
import torch

import pkhot
import scenes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


@pytest.mark.parametrize("cap", [60, 0])
@pytest.mark.parametrize("vis", [1.0, 0.05])
def test_viscosity_generic_list(ctx, oracle, cap, vis):
    sc = scenes.dam_break_small(seed=11, n_side=16)
    rng = np.random.default_rng(11)
    x0 = (sc.x + rng.uniform(-0.1, 0.1, sc.x.shape) * sc.spacing).astype(np.float32)
    v0 = rng.normal(0, 0.3, x0.shape).astype(np.float32)
    ri, re = oracle.neighbor_query(x0, sc.radius, sc.lo, sc.hi, cap)
    total = re.shape[0] if cap == 0 else x0.shape[0] * cap
    x, v = t(x0), t(v0)
    ctx.viscosity(x, v, t(ri).int(), t(re).int(), cap, total, vis, sc.radius, 5, sc.dt)
    ctx.check_status()
    vo = oracle.implicit_viscosity(x0, v0, ri, re, cap, vis, sc.radius, 5, sc.dt)
    vd = oracle.implicit_viscosity(x0, v0, ri, re, cap, vis, sc.radius, 5, sc.dt, dtype=np.float64)
    assert rel(v.cpu().numpy(), vo) < 1e-5
    assert rel(v.cpu().numpy(), vd) < 1e-5
    assert rel(vo, v0) > 1e-4  # the sweeps did change the field


def test_viscosity_properties(ctx, oracle):
    # a uniform field is a fixed point; an isolated particle (its list holds only
    # itself, skipped at r = 0) keeps its velocity; iterations = 0 is the identity
    sc = scenes.dam_break_small(seed=12, n_side=10)
    x0 = sc.x.copy()
    x0[0] = np.asarray(sc.hi, np.float32) - 0.001  # far from the block
    ri, re = oracle.neighbor_query(x0, sc.radius, sc.lo, sc.hi, 0)
    assert ri[1] - ri[0] == 1 and re[ri[0]] == 0
    v0 = np.tile(np.float32([0.3, -0.2, 0.1]), (x0.shape[0], 1))
    x, v = t(x0), t(v0)
    ctx.viscosity(x, v, t(ri).int(), t(re).int(), 0, re.shape[0], 1.0, sc.radius, 5, sc.dt)
    assert rel(v.cpu().numpy(), v0) < 1e-6
    v1 = np.random.default_rng(12).normal(0, 1, x0.shape).astype(np.float32)
    v = t(v1)
    ctx.viscosity(x, v, t(ri).int(), t(re).int(), 0, re.shape[0], 1.0, sc.radius, 5, sc.dt)
    assert np.array_equal(v.cpu().numpy()[0], v1[0])
    v = t(v1)
    ctx.viscosity(x, v, t(ri).int(), t(re).int(), 0, re.shape[0], 1.0, sc.radius, 0, sc.dt)
    assert np.array_equal(v.cpu().numpy(), v1)
    with pytest.raises(pkhot.PkError):
        ctx.viscosity(x, v, t(ri).int(), t(re).int(), 0, re.shape[0], -1.0, sc.radius, 5, sc.dt)


def oracle_step(oracle, sc, sdf, rnd, x, v, vis):
    x, v = oracle.sdf_constrain(x, v, sdf, rnd, 0.95, 0.0, sc.dt)
    ri, re = oracle.neighbor_query(x, sc.radius, sc.lo, sc.hi, sc.cap)
    x, v = oracle.integrate(x, v, sc.gravity, sc.dt)
    f, m = oracle.density_scaling(sc.spacing, sc.radius, sc.rest_density)
    x, v, _ = oracle.pbd_constrain(x, v, ri, re, sc.cap, sc.radius, f * m, sc.iterations, sc.dt)
    v = oracle.implicit_viscosity(x, v, ri, re, sc.cap, vis, sc.radius, 5, sc.dt)
    return x, v


def test_fused_step_with_viscosity_1_and_10(ctx, oracle):
    sc = scenes.dam_break_small(seed=13)
    x0 = sc.x.copy()
    x0[:, 1] -= 0.0052
    v0 = np.random.default_rng(13).normal(0, 0.05, x0.shape).astype(np.float32)
    ctx.boundary_set_box(sc.lo, sc.hi, sc.sdf_spacing, True)
    rnd = ctx.boundary_jitter(x0.shape[0]).cpu().numpy()
    sdf = oracle.sdf_box(sc.lo, sc.hi, sc.sdf_spacing, True)
    x, v = t(x0), t(v0)
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, 1000.0, 5, sc.dt), sc.gravity,
                           viscosity=1.0)
    xo, vo = x0, v0
    for step in range(10):
        ctx.pbf_step(x, v, prm)
        xo, vo = oracle_step(oracle, sc, sdf, rnd, xo, vo, 1.0)
        if step in (0, 9):
            ctx.check_status()
            assert rel(x.cpu().numpy(), xo) < 1e-4, step
            assert rel(v.cpu().numpy(), vo) < 1e-3, step


def test_fused_viscosity_equals_module_calls(ctx):
    # the fused stage on the solver rows against DensityPBD + ImplicitViscosity
    # through the generic entry points on the list NeighborQuery wrote
    sc = scenes.dam_break_small(seed=14, n_side=18)
    ctx.boundary_set_box(sc.lo, sc.hi, sc.sdf_spacing, True)
    x1, v1 = t(sc.x), t(sc.v)
    x2, v2 = t(sc.x), t(sc.v)
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, 1000.0, 5, sc.dt), sc.gravity,
                           viscosity=1.0, viscosity_iterations=5)
    for _ in range(3):
        ctx.pbf_step(x1, v1, prm)
        ctx.boundary_constrain(x2, v2, sc.dt)
        idx, el, tot = ctx.nq_build(x2, sc.radius, sc.lo, sc.hi, sc.cap)
        ctx.integrate(x2, v2, sc.gravity, sc.dt)
        ctx.pbd_solve(x2, v2, idx, el, sc.cap, tot, prm.pbd)
        ctx.viscosity(x2, v2, idx, el, sc.cap, tot, 1.0, sc.radius, 5, sc.dt)
    ctx.check_status()
    assert rel(x1.cpu().numpy(), x2.cpu().numpy().astype(np.float64)) < 1e-6
    assert rel(v1.cpu().numpy(), v2.cpu().numpy().astype(np.float64)) < 1e-5


def test_batched_with_viscosity_equals_single(ctx):
    b = scenes.batched_mix(seed=15, nscenes=5, n_min=200, n_max=3000)
    x0 = b.x.copy()
    x0[:, 1] -= 0.0052
    v0 = np.random.default_rng(15).normal(0, 0.05, x0.shape).astype(np.float32)
    sc0 = b.scenes[0]
    ctx.boundary_set_box(sc0.lo, sc0.hi, sc0.sdf_spacing, True)
    prm = pkhot.pbf_params(pkhot.nq_params(sc0.radius, sc0.lo, sc0.hi, sc0.cap),
                           pkhot.pbd_params(sc0.radius, sc0.spacing, sc0.rest_density, sc0.iterations, sc0.dt),
                           sc0.gravity, viscosity=1.0)
    xb, vb = t(x0), t(v0)
    off = torch.from_numpy(b.offsets.astype(np.int32)).cuda()
    for _ in range(2):
        ctx.pbf_step_batched(xb, vb, off, prm)
    ctx.check_status()
    xb, vb = xb.cpu().numpy(), vb.cpu().numpy()
    for s in range(len(b.scenes)):
        lo, hi = b.offsets[s], b.offsets[s + 1]
        xs, vs = t(x0[lo:hi]), t(v0[lo:hi])
        for _ in range(2):
            ctx.pbf_step(xs, vs, prm)
        ctx.check_status()
        assert np.array_equal(xs.cpu().numpy(), xb[lo:hi]), s
        assert np.array_equal(vs.cpu().numpy(), vb[lo:hi]), s
