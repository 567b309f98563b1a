"""The allocation-free DensityPBD solve (pk_pbd_solve_noalloc).

Some callers of this library cannot allocate device memory: an application
that manages the GPU's memory itself and forbids plugins to call cudaMalloc,
or a frame loop that cannot take cudaMalloc's synchronisation.  For them the
library keeps a fixed scratch array on the device and offers a solve that
needs no context.  This test checks it against the regular entry point
(pk_pbd_solve on the same, externally built list) on two calls in a row --
the second call reuses the scratch the first one left behind -- and that
sizes beyond the fixed scratch are refused.  The file is named so that
pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

import pkhot
import scenes

pytestmark = pytest.mark.gpu


def t(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def noalloc_solve(L, x, v, idx, el, cap, total, prm, rho):
    return L.pk_pbd_solve_noalloc(pkhot._ptr(x), pkhot._ptr(v), x.shape[0], pkhot._ptr(idx),
                                  pkhot._ptr(el), cap, total, ctypes.byref(prm), pkhot._ptr(rho),
                                  pkhot._stream())


def test_noalloc_matches_regular_solve_twice(oracle):
    L = pkhot.load()
    ctx = pkhot.Context(0)
    sc = scenes.dam_break_small(seed=11, n_side=20)
    v0 = np.random.default_rng(11).normal(0, 0.05, sc.x.shape).astype(np.float32)
    ri, re = oracle.neighbor_query(sc.x, sc.radius, sc.lo, sc.hi, sc.cap)
    idx, el = t(ri, np.int32), t(re, np.int32)
    total = sc.x.shape[0] * sc.cap
    prm = pkhot.pbd_params(sc.radius, sc.spacing, 1000.0, 5, sc.dt)
    xa, va = t(sc.x), t(v0)   # regular entry point
    xb, vb = t(sc.x), t(v0)   # allocation-free entry point
    rho_a = torch.zeros(sc.x.shape[0], device="cuda")
    rho_b = torch.zeros(sc.x.shape[0], device="cuda")
    for call in range(2):
        ctx.pbd_solve(xa, va, idx, el, sc.cap, total, prm, rho_a)
        assert noalloc_solve(L, xb, vb, idx, el, sc.cap, total, prm, rho_b) == pkhot.PK_OK
        torch.cuda.synchronize()
        assert rel(xb.cpu().numpy(), xa.cpu().numpy()) < 1e-5, call
        assert rel(vb.cpu().numpy(), va.cpu().numpy()) < 1e-4, call
        assert rel(rho_b.cpu().numpy(), rho_a.cpu().numpy()) < 1e-5, call
    ctx.close()


def test_noalloc_refuses_sizes_beyond_its_scratch():
    L = pkhot.load()
    nmax = L.pk_noalloc_max_particles()
    assert nmax == 131072
    x = torch.zeros((1, 3), device="cuda")
    prm = pkhot.pbd_params(0.0125, 0.005, 1000.0, 5, 1e-3)
    rc = L.pk_pbd_solve_noalloc(pkhot._ptr(x), pkhot._ptr(x), nmax + 1, pkhot._ptr(x), pkhot._ptr(x),
                                8, 0, ctypes.byref(prm), None, pkhot._stream())
    assert rc == pkhot.PK_ERR_CAPACITY
