"""The multi-process path on CPU: two gloo ranks shard a batch of images and meet only in their
timings (no data-path collective), as `bench.py --gpus N` runs one process per GPU."""
from __future__ import annotations

import os

import pytest
import torch
import torch.multiprocessing as mp

from structsplat_b200.replicas import max_over_ranks, shard_images, sum_over_ranks

SIZES = [(256, 256), (512, 512), (512, 768), (1024, 1024), (1536, 2048)] * 5 + [(64, 48)]


def test_shards_are_disjoint_cover_everything_and_balance():
    for world in (1, 2, 3, 4, 8):
        shards = [shard_images(SIZES, r, world) for r in range(world)]
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(SIZES)))
        loads = [sum(SIZES[i][0] * SIZES[i][1] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(h * w for h, w in SIZES)
    with pytest.raises(ValueError):
        shard_images(SIZES, 2, 2)


def test_without_process_group_values_pass_through():
    assert max_over_ranks([1.5, 2.0]) == [1.5, 2.0]
    assert sum_over_ranks([3]) == [3.0]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = shard_images(SIZES, rank, world)
        t = 10.0 + rank  # this rank's "time"
        mx = max_over_ranks([t, len(mine)])
        total = sum_over_ranks([len(mine)])
        out.put((rank, mine, mx, total))
    finally:
        torch.distributed.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce_timings():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, mx0, t0), (r1, s1, mx1, t1) = results
    assert set(s0).isdisjoint(s1) and sorted(s0 + s1) == list(range(len(SIZES)))
    assert mx0 == mx1 and mx0[0] == 11.0 and mx0[1] == max(len(s0), len(s1))
    assert t0 == t1 == [float(len(SIZES))]
