"""The frame autotuner (pk_ctx_autotune): its four trial frames run the
Jacobi passes at 128/256/512 threads per block and the neighbour sweep with 4,
8 and 16 particles per pass.  Those shapes change no result, so a tuned context
must step bit for bit like an untuned one, and it must settle on one of the
trial shapes."""
import numpy as np
import pytest
import torch

import pkhot
import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("viscosity", [0.0, 1.0])
def test_autotuned_frames_equal_untuned(viscosity):
    sc = scenes.dam_break_small(seed=21, n_side=24)
    x0 = sc.x.copy()
    x0[:, 1] -= 0.0052
    v0 = np.random.default_rng(21).normal(0, 0.05, x0.shape).astype(np.float32)
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt),
                           sc.gravity, viscosity=viscosity)
    out = []
    for tune in (False, True):
        ctx = pkhot.Context(0)
        ctx.boundary_set_box(sc.lo, sc.hi, sc.sdf_spacing, True)
        if tune:
            ctx.autotune(True)
            assert ctx.tuning()[2]
        x, v = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(v0.copy()).cuda()
        for _ in range(6):
            ctx.pbf_step(x, v, prm)
        ctx.check_status()
        pb, bp, active = ctx.tuning()
        if tune:
            assert not active and pb in (128, 256, 512) and bp in (4, 8, 16)
        else:
            assert (pb, bp, active) == (256, 8, False)
        out.append((x.cpu().numpy(), v.cpu().numpy()))
        ctx.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
