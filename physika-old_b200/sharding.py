"""Scene partitioning for batched frames on several GPUs (one process per GPU).

Independent scenes shard with no exchange: every rank steps its own subset in
one pk_pbf_step_batched call and nothing crosses NVLink during a frame.  The
subsets come from the longest-processing-time greedy rule on particle counts
(scenes in descending size, each to the least-loaded rank, ties to the lower
rank), which keeps the largest rank load within 4/3 of the optimum.
"""
import numpy as np


def partition_scenes(counts, world):
    """Per-rank lists of scene indices (ascending), covering every scene once."""
    counts = np.asarray(counts, np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(counts.shape[0]), key=lambda s: (-int(counts[s]), s))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for s in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(s)
        load[r] += int(counts[s])
    return [sorted(p) for p in parts]


def subset(x, v, offsets, scenes):
    """Concatenates the chosen scenes' particles; returns (x, v, offsets)."""
    offsets = np.asarray(offsets, np.int64)
    xs = [x[offsets[s]:offsets[s + 1]] for s in scenes]
    vs = [v[offsets[s]:offsets[s + 1]] for s in scenes]
    counts = np.array([offsets[s + 1] - offsets[s] for s in scenes], np.int64)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    if not scenes:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), off
    return np.concatenate(xs).astype(np.float32), np.concatenate(vs).astype(np.float32), off
