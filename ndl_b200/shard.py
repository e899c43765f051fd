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


# ---------------------------------------------------------------------------
# One volume too large for one GPU: slabs along the slowest axis
# ---------------------------------------------------------------------------
#
# A single volume (the 1024x1024x3x96 video, say) splits into contiguous slabs
# along its slowest axis (torch dim 0, ndl's last axis), one per rank.  The
# passes along the other axes act plane by plane, so only the pass along the
# slow axis needs data from other ranks: r = radius planes on each side, sent
# by the neighbouring ranks before the blur (the one exchange step).  At the
# volume's two ends the halo follows the border mode instead: Clamp repeats
# the end plane, Reflect mirrors the first/last r planes (mathHelpers.h:24),
# Wrap takes them from the rank at the other end (a ring).  Each rank then
# blurs its extended slab with the ordinary entry points and keeps its own
# planes; the halo planes' own outputs (which would need planes beyond the
# halo) are discarded.


def slab_bounds(n, world_size, rank):
    """[start, stop) of rank's slab of n planes (sizes differ by at most 1)."""
    base, extra = divmod(int(n), int(world_size))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def exchange_halo(local, r, border, group=None):
    """local: this rank's slab (torch dim 0 = the slow axis, contiguous).
    Returns the slab extended by r planes on each side: the neighbours'
    planes inside the volume, the border mode's planes outside it.  With
    torch.distributed uninitialised (or one rank) only the border planes are
    made.  Every slab needs at least r planes."""
    import torch
    import torch.distributed as dist

    from .image import BorderMode
    if r == 0:
        return local.contiguous()
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    n = local.shape[0]
    if n < r:
        raise ValueError("each slab needs at least r = %d planes (has %d)" % (r, n))
    ext = torch.empty((n + 2 * r,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    ext[r:r + n] = local
    wrap = int(border) == int(BorderMode.Wrap)
    first, last = rank == 0, rank == world - 1
    if world > 1:
        # gloo moves CPU tensors only; NCCL moves device tensors directly
        stage = dist.get_backend(group) == "gloo" and local.is_cuda
        send_lo = local[:r].contiguous()
        send_hi = local[n - r:].contiguous()
        recv_lo = torch.empty_like(send_lo)
        recv_hi = torch.empty_like(send_hi)
        if stage:
            send_lo, send_hi, recv_lo, recv_hi = (t.cpu() for t in (send_lo, send_hi, recv_lo, recv_hi))
        prev_rank = rank - 1 if not first else (world - 1 if wrap else None)
        next_rank = rank + 1 if not last else (0 if wrap else None)
        # message A: a slab's first planes, to the previous rank (its back
        # halo); message B: the last planes, to the next rank (its front
        # halo).  Sends A, B and receives A, B are posted in that order, so
        # that two ranks in a Wrap ring (each the other's previous and next)
        # match them without tags (NCCL matches per peer in posting order).
        TAG_A, TAG_B = 1, 2
        ops = []
        if prev_rank is not None:
            ops.append(dist.P2POp(dist.isend, send_lo, prev_rank, group, TAG_A))
        if next_rank is not None:
            ops.append(dist.P2POp(dist.isend, send_hi, next_rank, group, TAG_B))
        if next_rank is not None:
            ops.append(dist.P2POp(dist.irecv, recv_hi, next_rank, group, TAG_A))
        if prev_rank is not None:
            ops.append(dist.P2POp(dist.irecv, recv_lo, prev_rank, group, TAG_B))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if prev_rank is not None:
            ext[:r] = recv_lo.to(ext.device)
        if next_rank is not None:
            ext[r + n:] = recv_hi.to(ext.device)
    # the volume's own ends
    if first and not (wrap and world > 1):
        if wrap:
            ext[:r] = local[n - r:]
        elif int(border) == int(BorderMode.Reflect):
            ext[:r] = torch.flip(local[:r], dims=[0])
        else:
            ext[:r] = local[:1].expand((r,) + tuple(local.shape[1:]))
    if last and not (wrap and world > 1):
        if wrap:
            ext[r + n:] = local[:r]
        elif int(border) == int(BorderMode.Reflect):
            ext[r + n:] = torch.flip(local[n - r:], dims=[0])
        else:
            ext[r + n:] = local[n - 1:].expand((r,) + tuple(local.shape[1:]))
    return ext


def sharded_gaussian_blur_axes(local, sigmas, border, group=None, workspace=None, stream=None):
    """gaussian_blur_axes of a volume split into slabs along its slowest axis
    (torch dim 0 = the last ndl axis; sigmas in ndl axis order): one halo
    exchange, then the ordinary blur of the extended slab on this rank's
    GPU.  Returns this rank's slab of the result (the same values a single
    GPU computes for those planes)."""
    import torch

    from . import convolution as C
    from .image import Image
    st = float(sigmas[-1])
    r = C.gaussian_radius(st) if st > 0 else 0
    ext = exchange_halo(local, r, border, group)
    src = Image.from_tensor(ext)
    out = Image.empty(src.extent(), ext.dtype, device=ext.device)
    C.gaussian_blur_axes(src, out, list(sigmas), border, workspace=workspace, stream=stream)
    return out.tensor()[r:r + local.shape[0]]
