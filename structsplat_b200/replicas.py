"""One process per GPU without a data-path collective.

The path partitions by image: a batched fit of independent images needs no exchange between
GPUs, so N processes each fit a disjoint share of the images (``shard_images``) and only their
timings meet (``max_over_ranks``: a job is as slow as its slowest rank).  A single image is
replicated, not split.
"""
from __future__ import annotations

import torch


def shard_images(sizes, rank: int, world: int) -> list[int]:
    """Indices of the images rank ``rank`` of ``world`` fits: largest-first greedy assignment to
    the least-loaded rank by pixel count, so ranks get near-equal work; ties broken by index so
    every rank computes the same partition independently."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i][0] * sizes[i][1], i))
    load = [0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += sizes[i][0] * sizes[i][1]
    return [i for i in range(len(sizes)) if owner[i] == rank]


def max_over_ranks(values, device=None) -> list[float]:
    """Element-wise maximum of per-rank values (all ranks call it with the same length); the
    values themselves when no process group is initialised."""
    vals = [float(v) for v in values]
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.tolist()


def sum_over_ranks(values, device=None) -> list[float]:
    """Element-wise sum of per-rank values (e.g. images processed)."""
    vals = [float(v) for v in values]
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
    return t.tolist()
