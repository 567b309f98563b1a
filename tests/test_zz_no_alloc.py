"""The allocation-free DensityPBD solve (pk_pbd_solve_noalloc).

Some callers of this library cannot allocate device memory: an application
that manages the GPU's memory itself and forbids plugins to call cudaMalloc,
or a frame loop that cannot take cudaMalloc's synchronisation.  For them the
library keeps a fixed scratch array on the device and offers a solve that
needs no context.  These tests check it, on two calls in a row (the second
call reuses the scratch the first one left behind), against the regular entry
point (pk_pbd_solve on the same, externally built list) and against the CPU
restatement, on a capped list and on a CSR list; that a call after the first
changes the device's free memory by nothing; and that sizes beyond the fixed
scratch are refused.  The file is named so that pytest collects it last.
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


@pytest.mark.parametrize("cap", [60, 0])
def test_noalloc_matches_regular_solve_and_oracle_twice(oracle, cap):
    L = pkhot.load()
    ctx = pkhot.Context(0)
    sc = scenes.dam_break_small(seed=11, n_side=20)
    n = sc.x.shape[0]
    v0 = np.random.default_rng(11).normal(0, 0.05, sc.x.shape).astype(np.float32)
    ri, re = oracle.neighbor_query(sc.x, sc.radius, sc.lo, sc.hi, cap)
    idx, el = t(ri, np.int32), t(re, np.int32)
    total = n * cap if cap else re.shape[0]
    prm = pkhot.pbd_params(sc.radius, sc.spacing, 1000.0, 5, sc.dt)
    f, m = oracle.density_scaling(sc.spacing, sc.radius, 1000.0)
    xa, va = t(sc.x), t(v0)   # regular entry point
    xb, vb = t(sc.x), t(v0)   # allocation-free entry point
    xo, vo = sc.x.copy(), v0.copy()
    rho_a = torch.zeros(n, device="cuda")
    rho_b = torch.zeros(n, device="cuda")
    for call in range(2):
        ctx.pbd_solve(xa, va, idx, el, cap, total, prm, rho_a)
        assert noalloc_solve(L, xb, vb, idx, el, cap, total, prm, rho_b) == pkhot.PK_OK
        xo, vo, ro = oracle.pbd_constrain(xo, vo, ri, re, cap, sc.radius, f * m, 5, sc.dt)
        torch.cuda.synchronize()
        ctx.check_status()
        assert rel(xb.cpu().numpy(), xa.cpu().numpy()) < 1e-5, call
        assert rel(vb.cpu().numpy(), va.cpu().numpy()) < 1e-4, call
        assert rel(rho_b.cpu().numpy(), rho_a.cpu().numpy()) < 1e-5, call
        assert rel(xb.cpu().numpy(), xo) < 1e-5, call
        assert rel(vb.cpu().numpy(), vo) < 1e-4, call
        assert rel(rho_b.cpu().numpy(), ro) < 1e-5, call
    ctx.close()


def test_noalloc_allocates_nothing():
    L = pkhot.load()
    sc = scenes.dam_break_small(seed=12, n_side=16)
    n = sc.x.shape[0]
    # a simple CSR list: every particle its own only neighbour
    idx = torch.arange(n, dtype=torch.int32, device="cuda")
    el = torch.arange(n, dtype=torch.int32, device="cuda")
    x, v = t(sc.x), t(sc.v)
    rho = torch.zeros(n, device="cuda")
    prm = pkhot.pbd_params(sc.radius, sc.spacing, 1000.0, 5, sc.dt)
    assert noalloc_solve(L, x, v, idx, el, 0, n, prm, rho) == pkhot.PK_OK  # first call: address look-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert noalloc_solve(L, x, v, idx, el, 0, n, prm, rho) == pkhot.PK_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_refuses_sizes_beyond_its_scratch():
    L = pkhot.load()
    nmax = L.pk_noalloc_max_particles()
    assert nmax == 131072
    x = torch.zeros((1, 3), device="cuda")
    prm = pkhot.pbd_params(0.0125, 0.005, 1000.0, 5, 1e-3)
    rc = L.pk_pbd_solve_noalloc(pkhot._ptr(x), pkhot._ptr(x), nmax + 1, pkhot._ptr(x), pkhot._ptr(x),
                                8, 0, ctypes.byref(prm), None, pkhot._stream())
    assert rc == pkhot.PK_ERR_CAPACITY
