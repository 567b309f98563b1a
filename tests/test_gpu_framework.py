"""The C++ Framework mirror (reference class names: ParticleFluid,
PositionBasedFluidModel, NeighborQuery, DensityPBD, ParticleIntegrator,
StaticBoundary, ParticleElasticBody, ElasticityModule) driving the sm_100a
library through the C ABI, as a PhysIKA scene would: the same frames as the
direct C-ABI calls."""
import ctypes
import os

import numpy as np
import pytest
import torch

import pkhot
import scenes

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(pkhot.LIB_PATH), "libpkframework.so")


def fw():
    pkhot.load()
    L = ctypes.CDLL(LIB)
    f3 = ctypes.POINTER(ctypes.c_float)
    L.pkf_fluid_run.argtypes = [f3, f3, ctypes.c_int, f3, f3, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                                ctypes.c_int, f3, f3]
    L.pkf_elastic_run.argtypes = [f3, f3, ctypes.c_int, f3, f3, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                                  ctypes.c_int, f3, f3]
    return L


def fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def v3(t):
    return np.ascontiguousarray(np.asarray(t, np.float32))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("vis", [1.0, 0.0])
def test_particle_fluid_scene_equals_fused_frames(ctx, vis):
    # vis 1: the stock PositionBasedFluidModel (ImplicitViscosity with
    # viscosity 1); vis 0: the model without its viscosity module
    sc = scenes.dam_break_small(seed=6, n_side=14)
    x0 = sc.x.copy()
    x0[:, 1] -= 0.0052  # the boundary acts from the first frame
    v0 = np.random.default_rng(6).normal(0, 0.05, x0.shape).astype(np.float32)
    n, steps = x0.shape[0], 5
    xo, vo = np.zeros_like(x0), np.zeros_like(x0)
    rc = fw().pkf_fluid_run(fp(x0), fp(v0), n, fp(v3(sc.lo)), fp(v3(sc.hi)), sc.spacing, sc.radius, sc.cap,
                            sc.iterations, sc.dt, sc.sdf_spacing, 1, vis, steps, fp(xo), fp(vo))
    assert rc == 0
    ctx.boundary_set_box(sc.lo, sc.hi, sc.sdf_spacing, True)
    x, v = torch.from_numpy(x0).cuda(), torch.from_numpy(v0).cuda()
    prm = pkhot.pbf_params(pkhot.nq_params(sc.radius, sc.lo, sc.hi, sc.cap),
                           pkhot.pbd_params(sc.radius, sc.spacing, sc.rest_density, sc.iterations, sc.dt),
                           (0.0, -9.8, 0.0), viscosity=vis)
    for _ in range(steps):
        ctx.pbf_step(x, v, prm)
    ctx.check_status()
    assert rel(xo, x.cpu().numpy()) < 1e-6
    assert rel(vo, v.cpu().numpy()) < 1e-5
    assert np.all(xo[:, 1] > -0.5 * sc.spacing)


def test_particle_elastic_body_equals_module_calls(ctx):
    sc = scenes.elastic_bar(seed=7, dims=(12, 6, 6), cap=80)
    rng = np.random.default_rng(7)
    x0 = (sc.x + rng.uniform(-0.02, 0.02, sc.x.shape) * sc.spacing).astype(np.float32)
    v0 = rng.normal(0, 0.05, x0.shape).astype(np.float32)
    n, steps = x0.shape[0], 5
    xo, vo = np.zeros_like(x0), np.zeros_like(x0)
    rc = fw().pkf_elastic_run(fp(x0), fp(v0), n, fp(v3(sc.lo)), fp(v3(sc.hi)), sc.horizon, sc.cap, sc.dt, steps,
                              fp(xo), fp(vo))
    assert rc == 0
    x, v = torch.from_numpy(x0).cuda(), torch.from_numpy(v0).cuda()
    idx, el, tot = ctx.nq_build(x, sc.horizon, sc.lo, sc.hi, sc.cap)
    ctx.pd_init(x, idx, el, sc.cap, tot, sc.horizon)
    ctx.pd_set_bulk(torch.ones(n, device="cuda"))
    for _ in range(steps):
        ctx.integrate(x, v, (0.0, -9.8, 0.0), sc.dt)
        ctx.pd_solve(x, v, sc.horizon, 0.05, 0.1, 10, sc.dt)
    ctx.check_status()
    assert rel(xo, x.cpu().numpy()) < 1e-6
    assert rel(vo, v.cpu().numpy()) < 1e-5


def test_particle_fluid_from_obj_with_writer(ctx, tmp_path):
    # ParticleSystem::loadParticles(filename) + ParticleWriter frames: the
    # written frames equal the frames of the same scene started from the
    # same (parsed) positions
    sc = scenes.dam_break_small(seed=8, n_side=12)
    x0 = sc.x.copy()
    obj = tmp_path / "block.obj"
    obj.write_text("".join(f"v {a:.9g} {b:.9g} {c:.9g}\n" for a, b, c in x0))
    L = fw()
    f3 = ctypes.POINTER(ctypes.c_float)
    L.pkf_fluid_obj_run.argtypes = [ctypes.c_char_p, f3, f3, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                                    ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
    L.pkf_read_frame.argtypes = [ctypes.c_char_p, f3, f3, ctypes.c_int]
    out = str(tmp_path) + os.sep
    n = L.pkf_fluid_obj_run(str(obj).encode(), fp(v3(sc.lo)), fp(v3(sc.hi)), sc.spacing, sc.radius, sc.cap,
                            sc.iterations, sc.dt, sc.sdf_spacing, 1, 1.0, 4, out.encode(), b"frame_", 2)
    assert n == x0.shape[0]
    n_steps = {0: 2, 1: 4}
    for k, steps in n_steps.items():
        xf, cf = np.zeros_like(x0), np.ones(n, np.float32)
        assert L.pkf_read_frame(f"{out}frame_{k}.txt".encode(), fp(xf), fp(cf), n) == n
        assert np.all(cf == 0)
        xo, vo = np.zeros_like(x0), np.zeros_like(x0)
        v0 = np.zeros_like(x0)
        assert L.pkf_fluid_run(fp(x0), fp(v0), n, fp(v3(sc.lo)), fp(v3(sc.hi)), sc.spacing, sc.radius, sc.cap,
                               sc.iterations, sc.dt, sc.sdf_spacing, 1, 1.0, steps, fp(xo), fp(vo)) == 0
        assert np.array_equal(xf, xo), k
    assert not os.path.exists(f"{out}frame_2.txt")


def abi_elastoplastic(ctx, sc, x0, v0, frames, A, B, fracture):
    """ParticleElastoplasticBody::advance composed from C-ABI calls."""
    x, v = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(v0.copy()).cuda()
    n, h, dt = x0.shape[0], sc.horizon, sc.dt
    prm = pkhot.pbd_params(h, 0.005, 1000.0, 1, dt)
    idx, el, tot = ctx.nq_build(x, h, sc.lo, sc.hi, 0)
    ctx.pd_init(x, idx, el, 0, tot, h)
    ones = torch.ones(n, device="cuda")
    for _ in range(frames):
        ctx.integrate(x, v, (0.0, -9.8, 0.0), dt)
        idx, el, tot = ctx.nq_build(x, h, sc.lo, sc.hi, 0)
        ctx.pd_begin(x, h, 0.05, 0.1, dt)
        ctx.pd_compute_inverse_k(h)
        for _ in range(10):
            ctx.pd_enforce(x, h, 0.05, 0.1, dt)
            ctx.pbd_solve(x, v, idx, el, 0, tot, prm)
        ctx.pd_update_velocity(x, v, dt)
        idx, el, tot = ctx.nq_build(x, h, sc.lo, sc.hi, 0)
        if fracture:
            ctx.pd_fracture(x, h, A, B, 0.05, 0.1)
        else:
            ctx.pd_rotate_rest_shape(x, h)
            ctx.pd_set_bulk(ones)
            ctx.pd_apply_yielding(x, h, A, B, 0.05, 0.1)
            ctx.pd_reconstruct_rest_shape(x, idx, el, 0, tot, h, False)
        ctx.viscosity(x, v, idx, el, 0, tot, 1.0, h, 5, dt)
    ctx.check_status()
    return x.cpu().numpy(), v.cpu().numpy()


@pytest.mark.parametrize("fracture", [0, 1])
def test_particle_elastoplastic_body_equals_module_calls(ctx, oracle, fracture):
    sc = scenes.elastic_bar(seed=9, dims=(12, 6, 6), cap=0)
    rng = np.random.default_rng(9)
    x0 = (sc.x + rng.uniform(-0.02, 0.02, sc.x.shape) * sc.spacing).astype(np.float32)
    v0 = rng.normal(0, 0.05, x0.shape).astype(np.float32)
    v0[:, 0] += np.float32(0.5) * (x0[:, 1] - x0[:, 1].mean()) / np.float32(sc.spacing * 6)
    n, steps = x0.shape[0], 3
    L = fw()
    f3 = ctypes.POINTER(ctypes.c_float)
    L.pkf_elastoplastic_run.argtypes = [f3, f3, ctypes.c_int, f3, f3, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                        ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int, f3, f3]
    xo, vo = np.zeros_like(x0), np.zeros_like(x0)
    c = 1e-3 if fracture else 1e-4
    assert L.pkf_elastoplastic_run(fp(x0), fp(v0), n, fp(v3(sc.lo)), fp(v3(sc.hi)), sc.horizon, sc.dt, fracture,
                                   c, 60.0, 0, steps, fp(xo), fp(vo)) == 0
    A, B = oracle.drucker_prager(c, 60.0 / 180.0)
    xa, va = abi_elastoplastic(ctx, sc, x0, v0, steps, A, B, fracture)
    assert rel(xo, xa) < 1e-6
    assert rel(vo, va) < 1e-5
