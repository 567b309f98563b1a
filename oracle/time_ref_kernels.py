"""Device time of the reference's OWN hot-path kernels on the headline
workload (test infrastructure: a measurement recipe, not part of the product).

oracle/_ref/pkref_driver (`make -C oracle refk REF=<reference checkout>`)
compiles PhysIKA's GridHash.cu, NeighborQuery.cu, SummationDensity.cu,
DensityPBD.cu and ParticleIntegrator.cu unmodified and launches their kernels
as the reference's host methods do.  Its `pbf` command runs
PositionBasedFluidModel frames (query on the frame's start positions,
integrate, DensityPBD iterations, velocity update; no boundary, no
viscosity).  The driver's own checks between launches (host sums of the grid
counts, see oracle/refk/refk_grid.cu) make its wall clock meaningless, so the
frame's cost is taken as the sum of the kernels' device times from an ncu
launch list (one metric, one pass per launch).

    python oracle/time_ref_kernels.py write <in.bin> [frames]
    oracle/_ref/pkref_driver pbf <in.bin> <out.bin> &&
    ncu --metrics gpu__time_duration.sum --clock-control none --csv \\
        --log-file <launches.csv> oracle/_ref/pkref_driver pbf <in.bin> <out.bin>
    python oracle/time_ref_kernels.py summarise <launches.csv> [frames]

The input is the bench's headline scene (128^3 jittered lattice, 2,097,152
particles, spacing 0.0025, radius 0.00625, cap 64, 5 iterations, dt 5e-4),
at rest.
"""
import collections
import csv
import io
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "physika-old_b200"))

# kernel name -> stage of the frame
STAGES = {
    "K_CalculateParticleNumber": "grid hash", "K_ConstructHashTable": "grid hash",
    "K_ComputeNeighborFixed": "neighbour query",
    "K_UpdateVelocity": "integrate", "K_UpdatePosition": "integrate / position update",
    "K_ComputeDensity": "density", "K_ComputeLambdas": "lambda", "K_ComputeDisplacement": "displacement",
    "DP_UpdateVelocity": "velocity update",
}


def write(path, frames=3):
    import scenes
    sc = scenes.dam_break_2m(seed=0)
    x = np.ascontiguousarray(sc.x, np.float32)
    v = np.zeros_like(x)
    n = x.shape[0]
    head = np.asarray([n, sc.cap, sc.iterations, frames, 0], np.int32).tobytes()
    prm = np.asarray([sc.radius, sc.spacing, sc.rest_density, sc.dt, *sc.gravity, *sc.lo, *sc.hi], np.float32)
    with open(path, "wb") as f:
        f.write(head + prm.tobytes() + x.tobytes() + v.tobytes())
    print(f"wrote {path}: {n} particles, {frames} frames")


def summarise(csv_path, frames=3):
    txt = open(csv_path).read().splitlines()
    start = next(k for k, l in enumerate(txt) if l.startswith('"ID"'))
    per = collections.defaultdict(float)
    other = collections.defaultdict(float)
    count = collections.Counter()
    for r in csv.DictReader(io.StringIO("\n".join(txt[start:]))):
        if r["Metric Name"] != "gpu__time_duration.sum":
            continue
        name = r["Kernel Name"].split("(")[0].split("<")[0].replace("void ", "").split("::")[-1]
        ns = float(r["Metric Value"].replace(",", ""))
        count[name] += 1
        stage = STAGES.get(name)
        if stage:
            per[stage] += ns
        else:
            other[name] += ns  # the reduction and scan kernels of the grid hash
    total = sum(per.values()) + sum(other.values())
    print(f"frames: {frames}; kernel launches: {sum(count.values())}")
    for k, t in sorted(list(per.items()) + [(f"grid hash: {k}", t) for k, t in other.items()], key=lambda kv: -kv[1]):
        print(f"  {k:40s} {t / 1e6 / frames:9.3f} ms per frame")
    print(f"  {'total':40s} {total / 1e6 / frames:9.3f} ms per frame")


if __name__ == "__main__":
    if len(sys.argv) >= 3 and sys.argv[1] == "write":
        write(sys.argv[2], int(sys.argv[3]) if len(sys.argv) > 3 else 3)
    elif len(sys.argv) >= 3 and sys.argv[1] == "summarise":
        summarise(sys.argv[2], int(sys.argv[3]) if len(sys.argv) > 3 else 3)
    else:
        raise SystemExit(__doc__)
