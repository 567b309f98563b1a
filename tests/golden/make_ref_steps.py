"""Generates tests/golden/ref_steps.npz: neighbour lists and particle states
produced by the reference's OWN hot-path kernels, run on a GPU by
oracle/_ref/pkref_driver (`make -C oracle refk REF=<reference checkout>`).

The driver compiles PhysIKA's NeighborQuery.cu, GridHash.cu,
SummationDensity.cu, DensityPBD.cu, ParticleIntegrator.cu and
ElasticityModule.cu from the reference sources, unmodified, and launches their
kernels as the reference's host methods do (oracle/refk/). These fixtures pin
the control flow of the CPU restatement (27-cell walk and cap selection,
Jacobi structure and scatter semantics, bond projection), beside the
arithmetic that tests/golden/ref_math.npz already pins.

Cases (inputs seeded, numpy PCG64, stored beside the outputs; particle counts
are multiples of 64, see oracle/refk/refk.h):
  nq_dyn:   one dynamic (uncapped, CSR) query, 12^3 jittered lattice with the
            32,768-particle dam break's spacing and radius.
  pbf_c0:   10 PositionBasedFluidModel frames (query on the frame's start
            positions, integrate, 5 DensityPBD iterations, velocity update; no
            viscosity, no boundary) of a 12^3 block with the 32k dam break's
            parameters (spacing 0.005, radius 0.0125, cap 60, dt 1e-3).
  pbf_c1:   the same with the 2M dam break's parameters (spacing 0.0025,
            radius 2.5 spacing, cap 64, dt 5e-4).
  pbf_dense: the 32k dam break's parameters on a lattice compressed to 0.85
            spacing, so every interior particle is over-dense and the
            density constraint does large corrections.
  pd_c2:    10 ParticleElasticBody steps (integrate, ElasticityModule with 10
            projection iterations) of a 16x8x8 block with the elastic bar's
            spacing 0.004, horizon 3 spacing, cap 80, per-particle bulk
            stiffness U[0.8, 1.2] 1e4, mu 0.05, lambda 0.1, initial velocities
            N(0, 0.05^2); lattice jittered by 0.1 spacing so the cap's nearest
            80 are not decided by exact ties.
For each case <c>: <c>_x0, <c>_v0 (inputs), <c>_params; after steps 1 and 10:
<c>_s<k>_x, _v (and _rho, the last iteration's density, for PBF) and, for
PBF, the step's list as sorted rows: <c>_s<k>_cnt (per-particle count) and
<c>_s<k>_ids (rows concatenated, each sorted ascending). PD adds the rest
shape (rest_cnt, rest_ids sorted, rest_idx/rest_pos in the reference's
slot order) and K^-1 at t0 (invk, row-major 3x3 per particle).

Run on a machine with a GPU:
    python tests/golden/make_ref_steps.py [--out PATH]
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "pkref_driver")
sys.path.insert(0, os.path.join(ROOT, "physika-old_b200"))
import scenes  # noqa: E402

DUMPS = (1, 10)
STEPS = 10


def i32(*v):
    return np.asarray(v, np.int32).tobytes()


def f32(*v):
    return np.asarray(v, np.float32).tobytes()


def sorted_rows(index, elements, cap, n):
    cnt = np.empty(n, np.int32)
    rows = []
    for i in range(n):
        if cap > 0:
            r = elements[i * cap: i * cap + index[i]]
        else:
            end = index[i + 1] if i + 1 < n else elements.shape[0]
            r = elements[index[i]:end]
        cnt[i] = r.shape[0]
        rows.append(np.sort(r))
    return cnt, np.concatenate(rows).astype(np.int32)


class Reader:
    def __init__(self, path):
        self.b = open(path, "rb").read()
        self.o = 0

    def take(self, dtype, count):
        a = np.frombuffer(self.b, dtype, count, self.o).copy()
        self.o += a.nbytes
        return a

    def list(self, n, cap):
        total = int(self.take(np.int32, 1)[0])
        index = self.take(np.int32, n)
        el = self.take(np.int32, total)
        return index, el, total

    def done(self):
        assert self.o == len(self.b), (self.o, len(self.b))


def run(cmd, payload, tmp):
    pin, pout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
    with open(pin, "wb") as f:
        f.write(payload)
    subprocess.run([DRIVER, cmd, pin, pout], check=True, stdout=subprocess.DEVNULL)
    return Reader(pout)


def fluid_block(n_side, spacing, jitter, seed, origin):
    return scenes.lattice(n_side, n_side, n_side, spacing, jitter, seed, origin=origin)


def case_nq(out, tmp, seed):
    x = fluid_block(12, 0.005, 0.1, seed, (0.4, 0.4, 0.4))
    n, h, lo, hi = x.shape[0], 0.0125, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)
    r = run("nq", i32(n, 0) + f32(h) + f32(*lo) + f32(*hi) + x.tobytes(), tmp)
    index, el, _ = r.list(n, 0)
    r.done()
    out["nq_dyn_x0"] = x
    out["nq_dyn_params"] = np.array([h, *lo, *hi], np.float32)
    out["nq_dyn_cnt"], out["nq_dyn_ids"] = sorted_rows(index, el, 0, n)


def case_pbf(out, tmp, tag, x, spacing, h, cap, dt, lo, hi, iters=5, rho0=1000.0, g=(0.0, -9.8, 0.0)):
    n = x.shape[0]
    v = np.zeros_like(x)
    payload = (i32(n, cap, iters, STEPS, len(DUMPS)) + f32(h, spacing, rho0, dt) + f32(*g) + f32(*lo)
               + f32(*hi) + i32(*DUMPS) + x.tobytes() + v.tobytes())
    r = run("pbf", payload, tmp)
    factor, mass = r.take(np.float32, 2)
    out[f"{tag}_x0"], out[f"{tag}_v0"] = x, v
    out[f"{tag}_params"] = np.array([n, cap, iters, STEPS, h, spacing, rho0, dt, *g, *lo, *hi], np.float64)
    out[f"{tag}_factor_mass"] = np.array([factor, mass], np.float32)
    for k in DUMPS:
        assert int(r.take(np.int32, 1)[0]) == k
        out[f"{tag}_s{k}_x"] = r.take(np.float32, 3 * n).reshape(n, 3)
        out[f"{tag}_s{k}_v"] = r.take(np.float32, 3 * n).reshape(n, 3)
        out[f"{tag}_s{k}_rho"] = r.take(np.float32, n)
        index, el, _ = r.list(n, cap)
        out[f"{tag}_s{k}_cnt"], out[f"{tag}_s{k}_ids"] = sorted_rows(index, el, cap, n)
    r.done()


def case_pd(out, tmp, seed):
    tag = "pd_c2"
    s = 0.004
    x = scenes.lattice(16, 8, 8, s, 0.1, seed, origin=(0.1, 0.1, 0.1))
    n = x.shape[0]
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    bulk = rng.uniform(0.8e4, 1.2e4, n).astype(np.float32)
    v = rng.normal(0.0, 0.05, (n, 3)).astype(np.float32)
    horizon, cap, iters, mu, lam, dt = 3 * s, 80, 10, 0.05, 0.1, 1e-3
    g, lo, hi = (0.0, -9.8, 0.0), (0.0, 0.0, 0.0), (0.3, 0.3, 0.3)
    payload = (i32(n, cap, iters, STEPS, len(DUMPS)) + f32(horizon, mu, lam, dt) + f32(*g) + f32(*lo)
               + f32(*hi) + i32(*DUMPS) + x.tobytes() + v.tobytes() + bulk.tobytes())
    r = run("pd", payload, tmp)
    index, el, total = r.list(n, cap)
    rest_idx = r.take(np.int32, total)
    rest_pos = r.take(np.float32, 3 * total).reshape(total, 3)
    invk = r.take(np.float32, 9 * n).reshape(n, 3, 3)
    out[f"{tag}_x0"], out[f"{tag}_v0"], out[f"{tag}_bulk"] = x, v, bulk
    out[f"{tag}_params"] = np.array([n, cap, iters, STEPS, horizon, mu, lam, dt, *g, *lo, *hi], np.float64)
    out[f"{tag}_nbr_cnt"], out[f"{tag}_nbr_ids"] = sorted_rows(index, el, cap, n)
    # the rest shape in the reference's slot order (self first), cap-strided
    cnt = index.copy()
    keep = np.concatenate([np.arange(i * cap, i * cap + cnt[i]) for i in range(n)])
    out[f"{tag}_rest_cnt"] = cnt
    out[f"{tag}_rest_idx"] = rest_idx[keep]
    out[f"{tag}_rest_pos"] = rest_pos[keep]
    out[f"{tag}_invk"] = invk
    for k in DUMPS:
        assert int(r.take(np.int32, 1)[0]) == k
        out[f"{tag}_s{k}_x"] = r.take(np.float32, 3 * n).reshape(n, 3)
        out[f"{tag}_s{k}_v"] = r.take(np.float32, 3 * n).reshape(n, 3)
    r.done()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_steps.npz"))
    ap.add_argument("--seed", type=int, default=20261)
    a = ap.parse_args()
    if not os.path.exists(DRIVER):
        raise SystemExit("oracle/_ref/pkref_driver is missing: run `make -C oracle refk REF=<checkout>`")
    out = {"seed": np.int64(a.seed)}
    with tempfile.TemporaryDirectory() as tmp:
        case_nq(out, tmp, a.seed)
        unit = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
        case_pbf(out, tmp, "pbf_c0", fluid_block(12, 0.005, 0.1, a.seed + 10, (0.4, 0.4, 0.4)),
                 0.005, 0.0125, 60, 1e-3, *unit)
        case_pbf(out, tmp, "pbf_c1", fluid_block(12, 0.0025, 0.1, a.seed + 11, (0.5, 0.4, 0.4)),
                 0.0025, 0.00625, 64, 5e-4, (0.0, 0.0, 0.0), (2.0, 1.0, 1.0))
        case_pbf(out, tmp, "pbf_dense", fluid_block(12, 0.85 * 0.005, 0.1, a.seed + 12, (0.4, 0.4, 0.4)),
                 0.005, 0.0125, 60, 1e-3, *unit)
        case_pd(out, tmp, a.seed + 20)
    np.savez_compressed(a.out, **out)
    print(f"wrote {a.out} ({os.path.getsize(a.out)} bytes)")


if __name__ == "__main__":
    main()
