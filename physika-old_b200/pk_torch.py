"""torch.autograd.Function over the differentiable rollouts of the C ABI.

PdRollout.apply(x0, v0, bulk, ctx, settings) runs `steps` ElasticityModule
steps (integration + projection) on the sm_100a library and returns x_T; its
backward calls the hand-written adjoint (pk_pd_rollout_backward), which
replays the rollout from checkpoints and returns dL/dx0, dL/dv0 and dL/dbulk.
The context must have been initialised with pd_init on the rest shape; bond
breaking is not differentiable and is off.

PbdRollout.apply(x0, v0, ctx, params, steps, checkpoint_every) runs `steps`
DensityPBD frames (list, integration, Jacobi solve, velocity update; no
boundary, no viscosity) and returns (x_T, v_T); its backward calls
pk_pbd_rollout_backward and returns dL/dx0 and dL/dv0.

float32 and float64 tensors are supported (the float64 path is the reference
for gradient checks).

Both Functions call the library through its pybind11 layer (lib/_pkbind*.so,
csrc/pk_pybind.cpp), which checks the tensors and passes torch's current
stream; importing this module fails when that layer is not built.
"""
import ctypes
import importlib.util
import os
from dataclasses import dataclass

import torch


def _load_pkbind():
    import sysconfig
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                        "_pkbind" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built (run __graft_entry__.build())")
    import pkhot
    pkhot.load()  # libpkhot.so first, so the layer binds the same instance
    spec = importlib.util.spec_from_file_location("_pkbind", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


_pkbind = _load_pkbind()


def _handle(pk_ctx):
    return int(pk_ctx.h.value)


@dataclass
class RolloutSettings:
    horizon: float
    mu: float = 0.05
    lam: float = 0.1
    iterations: int = 10
    dt: float = 1e-3
    steps: int = 200
    checkpoint_every: int = 20
    gravity: tuple = (0.0, -9.8, 0.0)


class PdRollout(torch.autograd.Function):
    @staticmethod
    def forward(fctx, x0, v0, bulk, pk_ctx, s):
        x = x0.detach().clone().contiguous()
        v = v0.detach().clone().contiguous()
        b = bulk.detach().contiguous()
        h = _handle(pk_ctx)
        if x.dtype == torch.float32:
            _pkbind.pd_set_bulk(h, b)
            _pkbind.pd_rollout(h, x, v, s.horizon, s.mu, s.lam, s.iterations, s.dt, s.steps, s.checkpoint_every,
                               tuple(s.gravity))
        else:
            _pkbind.pd_rollout(h, x, v, s.horizon, s.mu, s.lam, s.iterations, s.dt, s.steps, s.checkpoint_every,
                               tuple(s.gravity), b)
        fctx.pk_ctx = pk_ctx
        fctx.bulk_dtype = bulk.dtype
        return x

    @staticmethod
    def backward(fctx, gx_t):
        gx, gv, gb = _pkbind.pd_rollout_backward(_handle(fctx.pk_ctx), gx_t.contiguous())
        return gx, gv, gb.to(fctx.bulk_dtype), None, None


def pd_rollout(x0, v0, bulk, pk_ctx, settings):
    """x_T of the rollout; differentiable in x0, v0 and bulk."""
    return PdRollout.apply(x0, v0, bulk, pk_ctx, settings)


class PbdRollout(torch.autograd.Function):
    @staticmethod
    def forward(fctx, x0, v0, pk_ctx, params, steps, checkpoint_every):
        x = x0.detach().clone().contiguous()
        v = v0.detach().clone().contiguous()
        _pkbind.pbd_rollout(_handle(pk_ctx), x, v, ctypes.addressof(params), steps, checkpoint_every)
        fctx.pk_ctx = pk_ctx
        return x, v

    @staticmethod
    def backward(fctx, gx_t, gv_t):
        gx, gv = _pkbind.pbd_rollout_backward(_handle(fctx.pk_ctx), gx_t.contiguous(), gv_t.contiguous())
        return gx, gv, None, None, None, None


def pbd_rollout(x0, v0, pk_ctx, params, steps, checkpoint_every=20):
    """(x_T, v_T) of the DensityPBD rollout; differentiable in x0 and v0."""
    return PbdRollout.apply(x0, v0, pk_ctx, params, steps, checkpoint_every)
