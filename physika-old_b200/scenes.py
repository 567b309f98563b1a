"""Seeded synthetic scenes with the shapes of the benchmark configurations.

Every scene is a jittered cubic lattice (numpy PCG64, seed given), the
stand-in for the reference's demo scenes (Examples/App_SingleFluid builds a
fluid block inside a StaticBoundary cube; App_Elasticity an elastic bar).
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class FluidScene:
    name: str
    x: np.ndarray            # (n, 3) float32
    v: np.ndarray            # (n, 3) float32
    spacing: float           # lattice spacing = DensityPBD sampling distance
    radius: float            # smoothing length = neighbour radius
    lo: tuple
    hi: tuple
    cap: int
    dt: float
    iterations: int = 5
    rest_density: float = 1000.0
    gravity: tuple = (0.0, -9.8, 0.0)
    sdf_spacing: float = 0.005
    steps: int = 100


@dataclass
class ElasticScene:
    name: str
    x: np.ndarray
    v: np.ndarray
    dims: tuple
    spacing: float
    horizon: float
    lo: tuple
    hi: tuple
    cap: int
    dt: float
    iterations: int = 10
    mu: float = 0.05
    lam: float = 0.1
    bulk: np.ndarray = field(default=None)
    break_stretch: float = 0.0
    steps: int = 500


def lattice(nx, ny, nz, spacing, jitter, seed, origin=(0.0, 0.0, 0.0)):
    """Lattice points at (index+1)*spacing + origin, jittered by U(-j, j)*spacing."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1)
    g = g.reshape(-1, 3).astype(np.float64)
    x = (g + 1.0) * spacing + np.asarray(origin, np.float64)
    if jitter > 0:
        x = x + rng.uniform(-jitter * spacing, jitter * spacing, size=x.shape)
    return x.astype(np.float32)


def dam_break_small(seed=0, n_side=32):
    """32^3 = 32,768 particles, spacing 0.005, +-0.1 spacing jitter, unit box,
    radius 0.0125, cap 60, dt 1e-3, 5 Jacobi iterations, 100 steps."""
    s = 0.005
    x = lattice(n_side, n_side, n_side, s, 0.1, seed)
    return FluidScene("dam_break_32k", x, np.zeros_like(x), s, 0.0125, (0.0, 0.0, 0.0),
                      (1.0, 1.0, 1.0), 60, 1e-3, steps=100)


def dam_break_2m(seed=0, n_side=128):
    """128^3 = 2,097,152 particles, spacing 0.0025, +-0.1 spacing jitter, 2x1x1
    box, radius 2.5 spacing, cap 64, dt 5e-4, 5 Jacobi iterations, 200 steps."""
    s = 0.0025
    x = lattice(n_side, n_side, n_side, s, 0.1, seed)
    return FluidScene("dam_break_2m", x, np.zeros_like(x), s, 2.5 * s, (0.0, 0.0, 0.0),
                      (2.0, 1.0, 1.0), 64, 5e-4, steps=200)


def elastic_bar(seed=0, dims=(256, 64, 32), spacing=0.004, cap=80, stiffness=(0.8e4, 1.2e4),
                steps=500):
    """Peridynamics bar: dims lattice, horizon 3 spacing, per-particle bulk
    stiffness U[stiffness] (seeded), 10 projection iterations."""
    x = lattice(*dims, spacing, 0.0, seed, origin=(0.1, 0.1, 0.1))
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    bulk = rng.uniform(stiffness[0], stiffness[1], size=x.shape[0]).astype(np.float32)
    ext = np.asarray(dims, np.float64) * spacing + 0.2
    return ElasticScene("elastic_bar", x, np.zeros_like(x), dims, spacing, 3.0 * spacing,
                        (0.0, 0.0, 0.0), tuple(float(e) for e in ext), cap, 1e-3, bulk=bulk,
                        break_stretch=0.02, steps=steps)


@dataclass
class BatchedScenes:
    name: str
    scenes: list             # FluidScene per scene (the configuration-0 parameters)
    x: np.ndarray            # (sum n_s, 3) float32, scenes concatenated
    v: np.ndarray
    offsets: np.ndarray      # (nscenes + 1,) int32


def batched_mix(seed=0, nscenes=256, n_min=1024, n_max=65536):
    """nscenes independent dam-break blocks, particle counts log-uniform in
    [n_min, n_max] (PCG64 seed), each a jittered lattice of about that many
    particles (dims a x a x c, a = round(n^(1/3))) in its own unit box with the
    32k dam break's parameters (spacing 0.005, radius 0.0125, cap 60, dt 1e-3,
    5 Jacobi iterations)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    target = np.round(np.exp(rng.uniform(np.log(n_min), np.log(n_max), nscenes))).astype(np.int64)
    scenes_, xs = [], []
    for s, n in enumerate(target):
        a = max(1, int(round(n ** (1.0 / 3.0))))
        c = max(1, int(round(n / (a * a))))
        base = dam_break_small(seed=seed * 100003 + s + 1, n_side=1)
        x = lattice(a, a, c, base.spacing, 0.1, seed * 100003 + s + 1)
        sc = FluidScene(f"scene{s}", x, np.zeros_like(x), base.spacing, base.radius, base.lo, base.hi,
                        base.cap, base.dt, steps=100)
        scenes_.append(sc)
        xs.append(x)
    counts = np.array([q.x.shape[0] for q in scenes_], np.int64)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    x = np.concatenate(xs).astype(np.float32)
    return BatchedScenes(f"batched_{nscenes}", scenes_, x, np.zeros_like(x), offsets)
