"""Batched frames: many independent scenes concatenated and stepped by one
pk_pbf_step_batched call must give, scene by scene, exactly what pk_pbf_step
gives for that scene alone (same neighbour sets, same sums in the same order,
the boundary jitter seeded by the id within the scene)."""
import numpy as np
import pytest
import torch

import pkhot
import scenes

pytestmark = pytest.mark.gpu


def t(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def params(sc):
    return pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                            pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt),
                            sc.gravity)


@pytest.mark.parametrize("seed", [1, 2])
def test_batched_equals_per_scene(ctx, seed):
    b = scenes.batched_mix(seed=seed, nscenes=12, n_min=100, n_max=3000)
    x0 = b.x.copy()
    x0[:, 1] -= 0.0052  # below the floor: the boundary (and its jitter) acts from the first frame
    v0 = np.random.default_rng(seed).normal(0, 0.05, x0.shape).astype(np.float32)
    sc0 = b.scenes[0]
    ctx.boundary_set_box(sc0.lo, sc0.hi, sc0.sdf_spacing, True)
    prm = params(sc0)
    xb, vb = t(x0), t(v0)
    off = t(b.offsets, np.int32)
    rho_b = torch.zeros(x0.shape[0], device="cuda")
    for _ in range(3):
        ctx.pbf_step_batched(xb, vb, off, prm, rho_b)
    ctx.check_status()
    xb, vb, rho_b = xb.cpu().numpy(), vb.cpu().numpy(), rho_b.cpu().numpy()
    for s in range(len(b.scenes)):
        lo, hi = b.offsets[s], b.offsets[s + 1]
        xs, vs = t(x0[lo:hi]), t(v0[lo:hi])
        rho = torch.zeros(hi - lo, device="cuda")
        for _ in range(3):
            ctx.pbf_step(xs, vs, prm, rho)
        ctx.check_status()
        assert np.array_equal(xs.cpu().numpy(), xb[lo:hi]), s
        assert np.array_equal(vs.cpu().numpy(), vb[lo:hi]), s
        assert np.array_equal(rho.cpu().numpy(), rho_b[lo:hi]), s


def test_tuned_batched_frames_equal_per_scene(ctx):
    # the autotuner's warm-up frame and four trial frames, the last with the Jacobi passes as a
    # resident grid walking the scene tiles; a few particles of one scene lie
    # outside every grid (their own tile range after all scenes)
    b = scenes.batched_mix(seed=3, nscenes=9, n_min=100, n_max=3000)
    x0 = b.x.copy()
    x0[b.offsets[4]:b.offsets[4] + 5] = 5.0
    v0 = np.random.default_rng(3).normal(0, 0.05, x0.shape).astype(np.float32)
    sc0 = b.scenes[0]
    prm = pkhot.pbf_params(pkhot.nq_params(sc0.radius, sc0.lo, sc0.hi, sc0.cap),
                           pkhot.pbd_params(sc0.radius, sc0.spacing, sc0.rest_density, sc0.iterations, sc0.dt),
                           sc0.gravity, boundary=False)
    tuned = pkhot.Context(0)
    tuned.autotune(True)
    xb, vb = t(x0), t(v0)
    off = t(b.offsets, np.int32)
    for _ in range(5):
        tuned.pbf_step_batched(xb, vb, off, prm)
    tuned.check_status()
    assert not tuned.tuning()[2]
    tuned.close()
    xb, vb = xb.cpu().numpy(), vb.cpu().numpy()
    for s in range(len(b.scenes)):
        lo, hi = b.offsets[s], b.offsets[s + 1]
        xs, vs = t(x0[lo:hi]), t(v0[lo:hi])
        for _ in range(5):
            ctx.pbf_step(xs, vs, prm)
        ctx.check_status()
        assert np.array_equal(xs.cpu().numpy(), xb[lo:hi]), s
        assert np.array_equal(vs.cpu().numpy(), vb[lo:hi]), s


def test_batched_arguments(ctx):
    x = t(np.zeros((4, 3)))
    sc = scenes.dam_break_small(n_side=2)
    with pytest.raises(pkhot.PkError) as e:
        ctx.pbf_step_batched(x, x.clone(), t(np.array([0], np.int32), np.int32), params(sc))
    assert e.value.code == pkhot.PK_ERR_ARG


@pytest.mark.parametrize("batched", [False, True])
def test_graph_frames_equal_eager_frames(batched):
    # pk_graph_capture runs one frame, records the next; every replay is that
    # frame again on the same buffers, bit for bit as eager frames
    b = scenes.batched_mix(seed=5, nscenes=6, n_min=200, n_max=2000)
    sc0 = b.scenes[0]
    x0 = b.x.copy() if batched else b.x[: b.offsets[1]].copy()
    v0 = np.random.default_rng(5).normal(0, 0.05, x0.shape).astype(np.float32)
    prm = params(sc0)
    off = t(b.offsets, np.int32) if batched else None
    c1, c2 = pkhot.Context(0), pkhot.Context(0)
    for c in (c1, c2):
        c.boundary_set_box(sc0.lo, sc0.hi, sc0.sdf_spacing, True)
    xe, ve = t(x0), t(v0)
    xg, vg = t(x0), t(v0)
    c2.graph_capture(xg, vg, prm, off)
    for k in range(4):
        if batched:
            c1.pbf_step_batched(xe, ve, off, prm)
        else:
            c1.pbf_step(xe, ve, prm)
        if k > 0:
            c2.graph_launch()
    torch.cuda.synchronize()
    c1.check_status()
    c2.check_status()
    assert np.array_equal(xe.cpu().numpy(), xg.cpu().numpy())
    assert np.array_equal(ve.cpu().numpy(), vg.cpu().numpy())
    c2.graph_release()
    with pytest.raises(pkhot.PkError) as e:
        c2.graph_launch()
    assert e.value.code == pkhot.PK_ERR_STATE
    c1.close()
    c2.close()
