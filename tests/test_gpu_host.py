"""pk_pbf_step_host: the frame on host arrays (copied in, stepped, copied
back on the call's stream) must equal pk_pbf_step on device arrays bit for
bit, for page-locked and pageable host memory, and its device copies must
grow when a larger scene arrives."""
import numpy as np
import pytest
import torch

import pkhot
import scenes

pytestmark = pytest.mark.gpu


def _scene(n_side, seed):
    sc = scenes.dam_break_small(seed=seed, n_side=n_side)
    x0 = sc.x.copy()
    x0[:, 1] -= 0.0052
    v0 = np.random.default_rng(seed).normal(0, 0.05, x0.shape).astype(np.float32)
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt),
                           sc.gravity)
    return sc, x0, v0, prm


@pytest.mark.parametrize("pinned", [True, False])
def test_host_frames_equal_device_frames(pinned):
    ctx_d, ctx_h = pkhot.Context(0), pkhot.Context(0)
    for n_side, seed in ((16, 3), (24, 4)):  # the second scene grows the device copies
        sc, x0, v0, prm = _scene(n_side, seed)
        for c in (ctx_d, ctx_h):
            c.boundary_set_box(sc.lo, sc.hi, sc.sdf_spacing, True)
        xd, vd = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(v0.copy()).cuda()
        xh, vh = torch.from_numpy(x0.copy()), torch.from_numpy(v0.copy())
        if pinned:
            xh, vh = xh.pin_memory(), vh.pin_memory()
        for _ in range(4):
            ctx_d.pbf_step(xd, vd, prm)
            ctx_h.pbf_step_host(xh, vh, prm)
        ctx_d.check_status()
        ctx_h.check_status()
        assert np.array_equal(xd.cpu().numpy(), xh.numpy())
        assert np.array_equal(vd.cpu().numpy(), vh.numpy())
    ctx_d.close()
    ctx_h.close()


def test_host_step_rejects_device_tensors():
    ctx = pkhot.Context(0)
    sc, x0, v0, prm = _scene(8, 5)
    with pytest.raises(ValueError):
        ctx.pbf_step_host(torch.from_numpy(x0).cuda(), torch.from_numpy(v0), prm)
    ctx.close()
