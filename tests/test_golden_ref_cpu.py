"""The CPU restatement against golden vectors of the reference's own compiled
arithmetic (tests/golden/ref_math.npz, made by tests/golden/make_ref_golden.py
with oracle/_ref/ref_math_probe on a B200): Vector3f::norm, on which every
neighbour decision d < h is taken (NeighborQuery.cu:266,357,536), and the
Spiky / Smooth / Corrected kernels (Kernel.h:29-142).  Bit-exact."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_math.npz")
TAGS = ("h0125", "h00625", "h012")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("tag", TAGS)
def test_norm_bit_exact(oracle, golden, tag):
    pairs, ref = golden["pairs_" + tag], golden["norm_" + tag][:, 0]
    got = oracle.dist3_many(pairs)
    bad = np.nonzero(got.view(np.uint32) != ref.view(np.uint32))[0]
    assert bad.size == 0, f"{bad.size} of {ref.size} norms differ, first pair {bad[:3]}"


@pytest.mark.parametrize("tag", TAGS)
def test_other_roundings_would_change_decisions(oracle, golden, tag):
    # the golden pairs separate the three ways of rounding x*x + y*y + z*z:
    # only the fused form the reference was compiled to decides every pair alike
    pairs, ref, h = golden["pairs_" + tag], golden["norm_" + tag][:, 0], golden["h_" + tag]
    try:
        for v in (0, 2):
            oracle.set_norm_variant(v)
            got = oracle.dist3_many(pairs)
            assert np.any((got < h) != (ref < h)), v
    finally:
        oracle.set_norm_variant(1)


@pytest.mark.parametrize("tag", TAGS)
def test_kernels_bit_exact(oracle, golden, tag):
    r, h, ref = golden["r_" + tag], golden["h_" + tag], golden["kern_" + tag]
    got = oracle.kernels(r, h)
    names = ("SpikyKernel::Weight", "SpikyKernel::Gradient", "SmoothKernel::Weight",
             "CorrectedKernel::Weight", "CorrectedKernel::WeightRR")
    for c, name in enumerate(names):
        bad = np.nonzero(got[:, c].view(np.uint32) != ref[:, c].view(np.uint32))[0]
        assert bad.size == 0, f"{name}: {bad.size} values differ, first r {r[bad[:3]]}"


def test_golden_pairs_are_borderline(golden):
    # half of each set lies within a few ulps of the radius
    for tag in TAGS:
        d, h = golden["norm_" + tag][:, 0], golden["h_" + tag]
        near = np.abs(d.astype(np.float64) - h) < 64 * np.spacing(np.float32(h))
        assert near.sum() > 1000, tag


def test_polar_decomposition_pinned_to_reference(oracle):
    # tests/golden/ref_polar.npz: the reference's own polarDecomposition (svd3,
    # McAdams et al.) run on a GPU by oracle/_ref/ref_math_probe
    # (tests/golden/make_ref_polar.py).  The restatement forms the same unique
    # products from a double-precision eigen-decomposition.
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_polar.npz"))
    # The reference's svd3 runs a fixed number of approximate Jacobi sweeps in
    # float; it is exact to rounding for most matrices and off by up to ~1e-3
    # (orthogonal entries) for a few with close singular values, where the
    # restatement stays exact.  Pinned: the median at rounding level, 99% of
    # the rotations within 1e-4, all within 0.05.
    R = oracle.polar_rotation(d["A_general"])
    err = np.abs(R - d["R_general"]).max(axis=1)  # rotations, reflections included
    assert np.median(err) < 2e-6 and np.percentile(err, 99) < 1e-4 and err.max() < 0.05
    # The clamped inverse of well-conditioned shape matrices (condition < 100,
    # full rank): the float SVD resolves the small singular values only to
    # ~1e-2 of the largest entry for a few percent of them.  Rank-deficient
    # inputs are left out: there the float SVD returns noise singular values
    # far above the clamp threshold and the reference's inverse is not
    # defined to better than its noise.
    thr = float(d["thr"])
    A = d["A_psd"].reshape(-1, 3, 3).astype(np.float64)
    w = np.linalg.eigvalsh(A)
    ok = (np.arange(A.shape[0]) < A.shape[0] // 2) & (w[:, 2] < 100 * np.maximum(w[:, 0], 1e-30))
    inv = oracle.clamped_inverse(d["A_psd"][ok], thr, 1.0)
    ref = d["Inv_psd"][ok].astype(np.float64)
    e2 = (np.abs(inv - ref) / np.abs(ref).max(axis=1, keepdims=True)).max(axis=1)
    assert ok.sum() > 500
    assert np.median(e2) < 1e-6 and np.percentile(e2, 90) < 1e-4 and e2.max() < 0.05
