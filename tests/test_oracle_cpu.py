"""CPU tests of the restatement (the checker): grid logic against brute force,
fixed-cap selection against the uncapped list, density normalisation, the
displacement scatter's momentum balance, and K^-1 on a lattice."""
import numpy as np
import pytest

import scenes
from nbr_util import rows


def brute_sets(x, h):
    d = np.sqrt(((x[:, None, :].astype(np.float64) - x[None, :, :]) ** 2).sum(-1))
    return d, [np.sort(np.nonzero(d[i] < h)[0]) for i in range(x.shape[0])]


@pytest.mark.parametrize("cap", [0, 20])
def test_neighbor_query_matches_brute_force(oracle, cap):
    sc = scenes.dam_break_small(seed=3, n_side=10)
    x = sc.x
    n = x.shape[0]
    idx, el = oracle.neighbor_query(x, sc.radius, sc.lo, sc.hi, cap)
    got = rows(idx, el, cap, n)
    d, ref = brute_sets(x, sc.radius)
    for i in range(n):
        if cap == 0:
            want = ref[i]
        else:
            order = np.argsort(d[i][ref[i]], kind="stable")
            want = np.sort(ref[i][order[:cap]])
        if not np.array_equal(got[i], want):
            # only pairs within float rounding of the radius / of each other may differ
            diff = np.setxor1d(got[i], want)
            assert np.all(np.abs(d[i][diff] - (sc.radius if cap == 0 else d[i][got[i]].max())) < 1e-7), i


def test_fixed_cap_is_cap_nearest_of_dynamic(oracle):
    sc = scenes.dam_break_small(seed=1, n_side=12)
    n = sc.x.shape[0]
    i0, e0 = oracle.neighbor_query(sc.x, sc.radius, sc.lo, sc.hi, 0)
    i1, e1 = oracle.neighbor_query(sc.x, sc.radius, sc.lo, sc.hi, 30)
    dyn, fix = rows(i0, e0, 0, n), rows(i1, e1, 30, n)
    for i in range(n):
        assert len(fix[i]) == min(30, len(dyn[i]))
        assert set(fix[i]) <= set(dyn[i])
        if len(dyn[i]) > 30:
            dmax = max(oracle.dist3(sc.x[i], sc.x[j]) for j in fix[i])
            rest = set(dyn[i]) - set(fix[i])
            assert all(oracle.dist3(sc.x[i], sc.x[j]) >= dmax for j in rest)


def test_self_in_list_and_outside_grid_dropped(oracle):
    x = np.array([[0.5, 0.5, 0.5], [0.505, 0.5, 0.5], [5.0, 5.0, 5.0]], np.float32)
    idx, el = oracle.neighbor_query(x, 0.0125, (0, 0, 0), (1, 1, 1), 0)
    r = rows(idx, el, 0, 3)
    assert list(r[0]) == [0, 1] and list(r[1]) == [0, 1]
    assert list(r[2]) == []  # outside the grid: not hashed, no valid cells around it


def test_rest_density_of_unjittered_lattice(oracle):
    s, h = 0.005, 0.0125
    x = scenes.lattice(12, 12, 12, s, 0.0, 0)
    idx, el = oracle.neighbor_query(x, h, (0, 0, 0), (1, 1, 1), 0)
    f, m = oracle.density_scaling(s, h, 1000.0)
    rho = oracle.summation_density(x, idx, el, 0, h, f * m)
    centre = np.all(np.abs(x - x.mean(0)) < 2 * s, axis=1)
    assert np.allclose(rho[centre], 1000.0, rtol=1e-4)


@pytest.mark.parametrize("cap", [0, 40])
def test_pbd_displacement_conserves_centroid(oracle, cap):
    sc = scenes.dam_break_small(seed=2, n_side=10)
    idx, el = oracle.neighbor_query(sc.x, sc.radius, sc.lo, sc.hi, cap)
    f, m = oracle.density_scaling(sc.spacing, sc.radius, 1000.0)
    x1, v1, rho = oracle.pbd_constrain(sc.x, sc.v, idx, el, cap, sc.radius, f * m, 5, sc.dt,
                                       dtype=np.float64)
    assert np.allclose(x1.astype(np.float64).mean(0), sc.x.astype(np.float64).mean(0), atol=1e-12)
    assert np.all(np.isfinite(x1)) and rho.max() > 100.0


def test_float_and_double_solver_agree(oracle):
    sc = scenes.dam_break_small(seed=4, n_side=10)
    idx, el = oracle.neighbor_query(sc.x, sc.radius, sc.lo, sc.hi, 60)
    f, m = oracle.density_scaling(sc.spacing, sc.radius, 1000.0)
    xf, _, _ = oracle.pbd_constrain(sc.x, sc.v, idx, el, 60, sc.radius, f * m, 5, sc.dt)
    xd, _, _ = oracle.pbd_constrain(sc.x, sc.v, idx, el, 60, sc.radius, f * m, 5, sc.dt,
                                    dtype=np.float64)
    assert np.linalg.norm(xf - xd) / np.linalg.norm(xd) < 1e-6


def test_integrator(oracle):
    x = np.zeros((4, 3), np.float32)
    v = np.ones((4, 3), np.float32)
    x1, v1 = oracle.integrate(x, v, (0, -9.8, 0), 0.01)
    assert np.allclose(v1[:, 1], 1 - 0.098) and np.allclose(x1[:, 1], 0.01 * (1 - 0.098))


def test_inverse_k_on_lattice_interior(oracle):
    sc = scenes.elastic_bar(dims=(8, 8, 8), cap=0)
    idx, el = oracle.neighbor_query(sc.x, sc.horizon, sc.lo, sc.hi, 0)
    ridx, rpos = oracle.pd_rest_shape(sc.x, idx, el, 0)
    inv = oracle.pd_inverse_k(idx, 0, el.shape[0], rpos, sc.horizon, dtype=np.float32)
    # self sits in slot 0 of every rest shape
    assert all(ridx[idx[i]] == i for i in range(sc.x.shape[0]))
    # interior K is isotropic: K^-1 is a multiple of the identity
    c = np.argmin(np.linalg.norm(sc.x - sc.x.mean(0), axis=1))
    K = inv[c]
    assert np.allclose(K, np.eye(3) * K[0, 0], rtol=1e-4, atol=1e-4 * abs(K[0, 0]))


def test_pd_static_lattice_stays_put(oracle):
    sc = scenes.elastic_bar(dims=(6, 6, 6), cap=0)
    idx, el = oracle.neighbor_query(sc.x, sc.horizon, sc.lo, sc.hi, 0)
    ridx, rpos = oracle.pd_rest_shape(sc.x, idx, el, 0)
    inv = oracle.pd_inverse_k(idx, 0, el.shape[0], rpos, sc.horizon)
    x1, v1 = oracle.pd_solve(sc.x, sc.v, idx, 0, el.shape[0], ridx, rpos, inv, sc.bulk, sc.horizon,
                             sc.mu, sc.lam, 10, sc.dt)
    assert np.max(np.abs(x1 - sc.x)) < 1e-5


def test_implicit_viscosity_properties(oracle):
    # ImplicitViscosity.cu:20-62: a uniform field is a fixed point, the sweep
    # is linear in v, and one sweep of a two-particle pair gives the closed form
    x = scenes.lattice(6, 6, 6, 0.005, 0.1, 3)
    ri, re = oracle.neighbor_query(x, 0.0125, (0, 0, 0), (1, 1, 1), 0)
    u = np.tile(np.float64([0.2, -0.1, 0.3]), (x.shape[0], 1))
    vu = oracle.implicit_viscosity(x, u, ri, re, 0, 1.0, 0.0125, 5, 1e-3, dtype=np.float64)
    assert np.allclose(vu, u, rtol=0, atol=1e-15)
    rng = np.random.default_rng(3)
    a, b = rng.normal(size=x.shape), rng.normal(size=x.shape)
    f = lambda v: oracle.implicit_viscosity(x, v, ri, re, 0, 1.0, 0.0125, 5, 1e-3, dtype=np.float64)
    assert np.allclose(f(2 * a - b), 2 * f(a) - f(b), rtol=0, atol=1e-12)
    xf = oracle.implicit_viscosity(x, a, ri, re, 0, 1.0, 0.0125, 5, 1e-3)
    assert np.abs(xf - f(a)).max() < 1e-5
    # two particles 0.006 apart: sum w v_j / sum w = v_other; b = dt vis / h
    x2 = np.float64([[0.5, 0.5, 0.5], [0.506, 0.5, 0.5]])
    v2 = np.float64([[1.0, 0, 0], [-1.0, 0, 0]])
    i2 = np.int32([0, 2])
    e2 = np.int32([0, 1, 0, 1])  # each list holds itself (r = 0 is skipped) and the other
    bb = 1e-3 * 1.0 / 0.0125
    got = oracle.implicit_viscosity(x2, v2, i2, e2, 0, 1.0, 0.0125, 1, 1e-3, dtype=np.float64)
    want = v2 / (1 + bb) + v2[::-1] * bb / (1 + bb)
    assert np.allclose(got, want, rtol=0, atol=1e-14)
