"""Generates tests/golden/ref_math.npz: golden values of the reference's own
device arithmetic on the hot path, computed on a GPU by oracle/_ref/ref_math_probe
(the reference's Vector3f::norm/normalize and Spiky/Smooth/Corrected kernels,
compiled by nvcc from the reference sources; see oracle/Makefile).

Inputs are seeded (numpy PCG64) and stored beside the outputs:
  pairs_<tag>: (n, 6) float32 particle pairs (a, b) for one radius h.  Half of
      them sit within a few ulps of |a - b| = h, where the rounding of the norm
      decides membership; the rest are spread over [0, 1.5 h).  Pair k is placed
      around its own lattice site 6 h apart from the others, so the pairs of one
      radius also form a scene whose neighbour lists are {self, partner?}.
  norm_<tag>: (n, 4) the reference's |a - b| and normalize(a - b).
  r_<tag>, kern_<tag>: radii in [0, 1.05 h] and the reference's SpikyKernel
      Weight/Gradient, SmoothKernel::Weight, CorrectedKernel Weight/WeightRR.

Run on a machine with a GPU after `make -C oracle ref`:
    python tests/golden/make_ref_golden.py [--out PATH]
"""
import argparse
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_math_probe")

# radius of each benchmark configuration: dam break 32k, dam break 2M, elastic bar
RADII = {"h0125": 0.0125, "h00625": 0.00625, "h012": 0.012}
PAIRS_PER_RADIUS = 4096
R_PER_RADIUS = 2048


def make_pairs(h, rng):
    n = PAIRS_PER_RADIUS
    side = int(np.ceil(n ** (1.0 / 3.0)))
    idx = np.stack(np.unravel_index(np.arange(n), (side, side, side)), -1).astype(np.float64)
    centre = 0.05 + (idx + 0.5) * 6.0 * h
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.empty(n)
    near = n // 2
    r[:near] = h * (1.0 + rng.uniform(-4e-7, 4e-7, near))  # a few ulps around h
    r[near:] = rng.uniform(0.0, 1.5 * h, n - near)
    a = centre + rng.uniform(-0.4 * h, 0.4 * h, (n, 3))
    b = a + d * r[:, None]
    return np.concatenate([a, b], axis=1).astype(np.float32)


def make_radii(h, rng):
    r = rng.uniform(0.0, 1.05 * h, R_PER_RADIUS)
    r[:8] = [0.0, h, np.nextafter(np.float32(h), np.float32(0)), 0.5 * h, 0.25 * h, 1e-7, h * 1.0000001, 0.999 * h]
    return r.astype(np.float32)


def run_probe(args):
    subprocess.run([PROBE] + args, check=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_math.npz"))
    ap.add_argument("--seed", type=int, default=20260)
    a = ap.parse_args()
    if not os.path.exists(PROBE):
        raise SystemExit("oracle/_ref/ref_math_probe is missing: run `make -C oracle ref` first")
    rng = np.random.Generator(np.random.PCG64(a.seed))
    out = {"seed": np.int64(a.seed)}
    with tempfile.TemporaryDirectory(dir=os.path.dirname(os.path.abspath(a.out))) as tmp:
        for tag, h in RADII.items():
            h32 = np.float32(h)
            pairs = make_pairs(float(h32), rng)
            pin, pout = os.path.join(tmp, "p.in"), os.path.join(tmp, "p.out")
            pairs.tofile(pin)
            run_probe(["pairs", pin, pout])
            out["pairs_" + tag] = pairs
            out["norm_" + tag] = np.fromfile(pout, np.float32).reshape(-1, 4)
            r = make_radii(float(h32), rng)
            rin, rout = os.path.join(tmp, "r.in"), os.path.join(tmp, "r.out")
            r.tofile(rin)
            run_probe(["kernels", float(h32).hex(), rin, rout])
            out["h_" + tag] = h32
            out["r_" + tag] = r
            out["kern_" + tag] = np.fromfile(rout, np.float32).reshape(-1, 5)
    np.savez_compressed(a.out, **out)
    print(f"wrote {a.out}")


if __name__ == "__main__":
    main()
