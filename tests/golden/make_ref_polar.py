"""Generates tests/golden/ref_polar.npz: the reference's own polarDecomposition
(Core/Algorithm/MatrixFunc.inl:81-98 on the vendored svd3, McAdams et al.
2011), computed on a GPU by oracle/_ref/ref_math_probe (built from the
reference sources by `make -C oracle ref`).

Inputs are seeded (numpy PCG64) and stored beside the outputs:
  A_general: (n, 9) float32 row-major matrices R1 diag(s) R2 with random
      rotations, singular values in [0.5, 2] (distinct), half of them with a
      reflection (det < 0): the deformation gradients EM_RotateRestShape
      decomposes (ElastoplasticityModule.cu:624-634).
  A_psd: (n, 9) symmetric positive semi-definite Q diag(w) Q^T with w spread
      over [1e-3, 1], or of rank 2 or 1 (w = 0 below the threshold): the shape
      matrices whose clamped inverse V D' U^T the plasticity and elasticity
      kernels form (ElastoplasticityModule.cu:442-458,624-629,
      ElasticityModule.cu:74-81).
  R_*, D_*, Inv_*: the probe's rotation, diagonal and clamped inverse
      (D' = 1/D above thr, 1 below).

Run on a machine with a GPU after `make -C oracle ref`:
    python tests/golden/make_ref_polar.py [--out PATH]
"""
import argparse
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_math_probe")
N = 2048
THR = 1.2e-6  # 1e-4 * h at the elastic bar's horizon (0.012)


def rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
        2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
        2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1).reshape(n, 3, 3)


def general(rng, n):
    s = np.sort(rng.uniform(0.5, 2.0, size=(n, 3)), axis=1)[:, ::-1]
    s[:, 1] = np.minimum(s[:, 1], s[:, 0] * 0.95)
    s[:, 2] = np.minimum(s[:, 2], s[:, 1] * 0.95)
    s[n // 2:, 2] *= -1.0  # reflections
    A = rotations(rng, n) @ (s[:, :, None] * rotations(rng, n))
    return A.astype(np.float32).reshape(n, 9)


def psd(rng, n):
    # eigenvalues over three decades (the float SVD resolves a small
    # eigenvalue only relative to the largest), a quarter of rank 2 and a
    # quarter of rank 1 (zero eigenvalues fall below the threshold)
    w = 10.0 ** rng.uniform(-3.0, 0.0, size=(n, 3))
    w[n // 2:3 * n // 4, 2] = 0.0
    w[3 * n // 4:, 1:] = 0.0
    Q = rotations(rng, n)
    A = Q @ (w[:, :, None] * np.transpose(Q, (0, 2, 1)))
    A = 0.5 * (A + np.transpose(A, (0, 2, 1)))
    return A.astype(np.float32).reshape(n, 9)


def run_probe(A):
    with tempfile.TemporaryDirectory() as d:
        fi, fo = os.path.join(d, "in.f32"), os.path.join(d, "out.f32")
        A.astype(np.float32).tofile(fi)
        subprocess.run([PROBE, "polar", repr(THR), fi, fo], check=True)
        out = np.fromfile(fo, np.float32).reshape(-1, 21)
    return out[:, :9], out[:, 9:12], out[:, 12:]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_polar.npz"))
    args = ap.parse_args()
    rng = np.random.Generator(np.random.PCG64(20261203))
    res = {"thr": np.float32(THR)}
    for tag, A in (("general", general(rng, N)), ("psd", psd(rng, N))):
        R, D, Inv = run_probe(A)
        res[f"A_{tag}"], res[f"R_{tag}"], res[f"D_{tag}"], res[f"Inv_{tag}"] = A, R, D, Inv
    np.savez_compressed(args.out, **res)
    print("wrote", args.out, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    main()
