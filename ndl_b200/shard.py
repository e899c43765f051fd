"""Sharding of independent instances across ranks (one process per GPU).

The batched workload is a set of independent images/volumes, so it shards
with no data-path collective: every rank computes the same deterministic
partition from the instances' cost estimates (voxels x taps per voxel) and
runs only its own share.  The only collective is the max of the per-rank
device times (the job's time), done with torch.distributed (NCCL on GPUs,
gloo in the CPU tests).
"""
from __future__ import annotations

import heapq


def instance_cost(extent, taps_per_axis):
    """Work estimate of one instance: elements x (sum of taps over its passes)."""
    n = 1
    for e in extent:
        n *= int(e)
    return n * max(1, sum(int(k) for k in taps_per_axis))


def partition(costs, world_size):
    """Longest-processing-time greedy partition: instances sorted by cost
    (ties by index), each to the currently lightest rank (ties by rank).
    Deterministic; returns one list of instance indices per rank."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world_size)]
    parts = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for p in parts:
        p.sort()
    return parts


def job_time_ms(local_ms, group=None, device=None):
    """Max over ranks of a per-rank device time (the time of the whole job)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(local_ms)
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
