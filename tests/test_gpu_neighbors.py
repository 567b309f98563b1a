"""NeighborQuery parity: the sm_100a list build against the CPU restatement,
compared as sorted per-particle sets (bit-exact), fixed and dynamic layouts,
plus the edge cases the reference's grid has (empty input, one particle,
particles outside the padded grid, coincident particles, overfull cells)."""
import numpy as np
import pytest
import torch

import scenes
from nbr_util import compare_capped, rows

pytestmark = pytest.mark.gpu


def gpu_query(ctx, x, h, lo, hi, cap):
    xt = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    idx, el, tot = ctx.nq_build(xt, h, lo, hi, cap)
    ctx.check_status()
    return idx.cpu().numpy(), el.cpu().numpy(), tot


def assert_same_lists(oracle, x, h, lo, hi, cap):
    n = x.shape[0]
    gi, ge, _ = gpu_query(pytest.ctx_handle, x, h, lo, hi, cap)
    ri, re = oracle.neighbor_query(x, h, lo, hi, cap)
    if cap == 0:
        assert np.array_equal(gi[:n], ri[:n]), "CSR offsets differ"
    else:
        assert np.array_equal(gi[:n], ri[:n]), "neighbour counts differ"
    ga, rb = rows(gi, ge, cap, n), rows(ri, re, cap, n)
    if cap == 0:
        bad = [i for i in range(n) if not np.array_equal(ga[i], rb[i])]
    else:
        bad = compare_capped(x, ga, rb, oracle.dist3, h)
    assert not bad, f"{len(bad)} particles with different neighbour sets, first {bad[:5]}"
    return ga


@pytest.fixture(autouse=True)
def _bind(ctx):
    pytest.ctx_handle = ctx


@pytest.mark.parametrize("cap", [60, 20, 0])
def test_dam_break_32k(oracle, cap):
    sc = scenes.dam_break_small(seed=0)
    assert_same_lists(oracle, sc.x, sc.radius, sc.lo, sc.hi, cap)


@pytest.mark.parametrize("cap", [64, 0])
def test_dam_break_2m_shape_small_block(oracle, cap):
    # the 2M scene's spacing, radius, box and cap on a 40^3 block
    sc = scenes.dam_break_2m(seed=5, n_side=40)
    assert_same_lists(oracle, sc.x, sc.radius, sc.lo, sc.hi, cap)


@pytest.mark.parametrize("cap", [60, 20])
def test_repeated_builds_with_moving_particles(oracle, cap):
    # the capped selection starts from each particle's previous tau: lists of
    # later frames on the same context (small moves, a large jump, a shuffled
    # caller order so the carried-over pivots belong to other particles) must
    # stay bit-exact
    sc = scenes.dam_break_small(seed=9, n_side=20)
    rng = np.random.default_rng(9)
    x = sc.x.copy()
    for step, amp in enumerate((0.0, 0.02, 0.05, 0.5, 0.01)):
        x = (x + rng.uniform(-amp, amp, x.shape) * sc.spacing).astype(np.float32)
        if step == 3:
            x = x[rng.permutation(x.shape[0])]
        assert_same_lists(oracle, x, sc.radius, sc.lo, sc.hi, cap)


def test_empty_and_single(ctx, oracle):
    for n in (0, 1):
        x = np.full((n, 3), 0.5, np.float32)
        gi, ge, tot = gpu_query(ctx, x, 0.0125, (0, 0, 0), (1, 1, 1), 8)
        if n == 1:
            assert gi[0] == 1 and ge[0] == 0


def test_outside_grid_and_coincident(oracle):
    rng = np.random.default_rng(7)
    x = rng.uniform(0.4, 0.45, size=(300, 3)).astype(np.float32)
    x[:40] = x[0]                      # 40 coincident particles (exact distance ties)
    x[40:50] = [5.0, 5.0, 5.0]         # far outside the padded grid: not hashed
    x[50:55] = [-0.02, 0.5, 0.5]       # in the padding cells: hashed
    x[55:60] = [-0.03, 0.5, 0.5]       # one cell outside: not hashed, still queries
    for cap in (0, 16, 80):
        assert_same_lists(oracle, x, 0.0125, (0, 0, 0), (1, 1, 1), cap)


def test_overfull_cells_capped(oracle):
    # a compressed cluster: 400 hits per particle, cap 64 selects among them
    rng = np.random.default_rng(9)
    x = rng.uniform(0.5, 0.508, size=(400, 3)).astype(np.float32)
    assert_same_lists(oracle, x, 0.0125, (0, 0, 0), (1, 1, 1), 64)


def test_dynamic_list_is_symmetric_at_scale(ctx):
    # size-independent property at the 2M scene's density: j in N(i) <=> i in N(j)
    sc = scenes.dam_break_2m(seed=1, n_side=64)
    gi, ge, tot = gpu_query(ctx, sc.x, sc.radius, sc.lo, sc.hi, 0)
    n = sc.x.shape[0]
    cnt = np.diff(np.r_[gi, tot])
    src = np.repeat(np.arange(n), cnt)
    fwd = src.astype(np.int64) * n + ge
    bwd = ge.astype(np.int64) * n + src
    assert np.array_equal(np.sort(fwd), np.sort(bwd))
    assert np.all(ge[gi] >= 0) and cnt.min() >= 1  # self is always present


@pytest.mark.parametrize("tag", ["h0125", "h00625", "h012"])
@pytest.mark.parametrize("cap", [0, 4])
def test_golden_pairs_decided_like_the_reference(ctx, tag, cap):
    # pairs within a few ulps of |a - b| = h, decided by the reference's own
    # compiled Vector3f::norm (tests/golden/ref_math.npz): each pair is
    # isolated, so a particle's list is itself plus its partner iff d < h
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_math.npz"))
    pairs, d, h = g["pairs_" + tag], g["norm_" + tag][:, 0], float(g["h_" + tag])
    x = pairs.reshape(-1, 3)
    hi = tuple(float(v) for v in x.max(0) + 0.1)
    gi, ge, _ = gpu_query(ctx, x, h, (0.0, 0.0, 0.0), hi, cap)
    got = rows(gi, ge, cap, x.shape[0])
    n = pairs.shape[0]
    want_pair = d < np.float32(h)
    bad = [k for k in range(n)
           if sorted(got[2 * k].tolist()) != ([2 * k, 2 * k + 1] if want_pair[k] else [2 * k])
           or sorted(got[2 * k + 1].tolist()) != ([2 * k, 2 * k + 1] if want_pair[k] else [2 * k + 1])]
    assert not bad, f"{len(bad)} of {n} pairs decided differently, first {bad[:5]}"
