"""The multi-process paths on CPU with the gloo backend (world size 2): the
scene partition of batched frames (every scene on exactly one rank, loads
balanced), and the bench's timing reduction (max over ranks after a barrier)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import scenes
from sharding import partition_scenes, subset


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch
        b = scenes.batched_mix(seed=0, nscenes=40, n_min=64, n_max=4096)
        counts = np.diff(b.offsets)
        mine = partition_scenes(counts, world)[rank]
        x, v, off = subset(b.x, b.v, b.offsets, mine)
        # the ranks' particle sets are exactly the scenes assigned to them
        assert off[-1] == counts[mine].sum() and x.shape[0] == off[-1]
        for k, s in enumerate(mine):
            assert np.array_equal(x[off[k]:off[k + 1]], b.x[b.offsets[s]:b.offsets[s + 1]])
        got = [None] * world
        dist.all_gather_object(got, mine)
        # timing reduction as bench.py does it
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            out.put((got, float(t.item()), counts.tolist()))
    finally:
        dist.destroy_process_group()


def test_partition_rules():
    counts = np.array([5, 9, 1, 7, 7, 3, 2, 8])
    parts = partition_scenes(counts, 3)
    flat = sorted(s for p in parts for s in p)
    assert flat == list(range(8))
    loads = [int(counts[p].sum()) for p in parts]
    assert max(loads) - min(loads) <= counts.max()
    assert partition_scenes(counts, 1) == [list(range(8))]
    assert partition_scenes(counts, 3) == parts  # deterministic
    with pytest.raises(ValueError):
        partition_scenes(counts, 0)


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got, tmax, counts = q.get(timeout=10)
    flat = sorted(s for part in got for s in part)
    assert flat == list(range(len(counts)))
    assert not set(got[0]) & set(got[1])
    loads = [sum(counts[s] for s in part) for part in got]
    assert max(loads) <= 1.34 * (sum(counts) / 2) + max(counts)
    assert tmax == 2.0
