"""Splitting the path over GPUs: one process per GPU, no collective on the
data path.

Every sample depends only on its pointing and the read-only map and beam, so
ranks work independently:

* :func:`sample_shard` -- contiguous, balanced sample ranges (a day's scan
  split across ranks keeps each rank's samples neighbours on the sky);
* :func:`detector_shards` -- detectors of uneven cost (scan length x beam
  pixels) assigned longest-first to the least-loaded rank;
* :func:`day_shard` -- whole days of the reference's day loop
  (gridint.py:311-333 hands days to worker processes) dealt round-robin;
* :func:`gather_shards` -- the one optional exchange: all ranks' (C, n_r)
  TOD pieces concatenated along samples, through ``torch.distributed``
  (NCCL for CUDA tensors, gloo on the CPU).
"""

from __future__ import annotations

import heapq

import torch

__all__ = ["sample_shard", "detector_shards", "day_shard", "gather_shards"]


def sample_shard(n, rank, world):
    """[start, stop) of rank ``rank``'s samples out of n; sizes differ by at most 1."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("need world >= 1, 0 <= rank < world and n >= 0")
    q, r = divmod(int(n), int(world))
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def detector_shards(costs, world):
    """Detector indices per rank: longest processing time first onto the
    currently least-loaded rank (ties: lower detector index first, then lower
    rank), each rank's list in increasing detector order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(v) for v in out]


def day_shard(start_day, end_day, rank, world):
    """Days start_day .. end_day - 1 dealt round-robin; this rank's list."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need world >= 1 and 0 <= rank < world")
    return list(range(int(start_day) + rank, int(end_day), world))


def gather_shards(local, n_total, group=None):
    """Concatenate every rank's (C, n_r) piece, the pieces of
    :func:`sample_shard` in rank order, into (C, n_total) on every rank."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    sizes = [sample_shard(n_total, r, world) for r in range(world)]
    width = max(b - a for a, b in sizes)
    C = local.shape[0]
    padded = torch.zeros((C, width), dtype=local.dtype, device=local.device)
    padded[:, :local.shape[1]] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p[:, :b - a] for p, (a, b) in zip(parts, sizes)], dim=1)
