"""Multi-process host logic of the sharded batched form, on CPU with gloo
(world size 2): both ranks derive the same disjoint, complete, balanced
partition, and the job time is the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from ndl_b200.shard import instance_cost, job_time_ms, partition


def test_partition_properties():
    costs = [instance_cost((s, s, s), (9, 9, 9)) for s in (32, 160, 64, 100, 40, 150, 90, 33)]
    parts = partition(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / 3 + max(costs)
    assert partition(costs, 3) == parts
    assert partition([], 2) == [[], []]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = partition(costs, world)
        mine = parts[rank]
        local = float(sum(costs[i] for i in mine)) / 1e6   # stands in for a measured time
        t = job_time_ms(local)
        q.put((rank, mine, t, parts))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_partition_and_job_time():
    costs = [instance_cost((s, s), (13, 13)) for s in range(64, 2048, 97)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (_, mine0, t0, parts0), (_, mine1, t1, parts1) = res
    assert parts0 == parts1
    assert sorted(mine0 + mine1) == list(range(len(costs))) and not set(mine0) & set(mine1)
    expect = max(sum(costs[i] for i in mine0), sum(costs[i] for i in mine1)) / 1e6
    assert abs(t0 - expect) < 1e-9 and abs(t1 - expect) < 1e-9


# -- slabs of one volume along its slowest axis: the halo exchange ----------

def _halo_worker(rank, world, port, vol, r, border, q):
    import torch.distributed as dist
    from ndl_b200.shard import exchange_halo, slab_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a, b = slab_bounds(vol.shape[0], world, rank)
        ext = exchange_halo(vol[a:b].clone(), r, border)
        q.put((rank, a, b, ext.numpy()))          # by value: outlives this process
    finally:
        dist.destroy_process_group()


def _expected_halo(vol, a, b, r, border):
    """The extended slab built directly from the whole volume with the
    border maps of mathHelpers.h:23-25."""
    import torch
    n = vol.shape[0]
    idx = []
    for t in range(a - r, b + r):
        if 0 <= t < n:
            idx.append(t)
        elif border == 1:                               # Wrap
            idx.append(t + n if t < 0 else t - n)
        elif border == 2:                               # Reflect
            idx.append(-t - 1 if t < 0 else 2 * n - t - 1)
        else:                                           # Clamp
            idx.append(0 if t < 0 else n - 1)
    return vol[torch.tensor(idx)]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_slab_halo_exchange_gloo(world, border):
    """Every rank's extended slab equals the volume's planes (border-mapped
    beyond its ends), for 2 ranks (each the other's neighbour on both sides
    under Wrap) and 3."""
    import torch
    vol = torch.arange(14 * 3 * 2, dtype=torch.float32).reshape(14, 3, 2)
    r = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_halo_worker, args=(k, world, port, vol, r, border, q)) for k in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, a, b, ext in res:
        assert torch.equal(torch.from_numpy(ext), _expected_halo(vol, a, b, r, border)), (rank, border)


def test_slab_bounds_and_single_rank_halo():
    import torch
    from ndl_b200.shard import exchange_halo, slab_bounds
    spans = [slab_bounds(10, 3, k) for k in range(3)]
    assert spans == [(0, 4), (4, 7), (7, 10)]
    vol = torch.arange(6, dtype=torch.float32).reshape(6, 1)
    for border in (0, 1, 2):
        assert torch.equal(exchange_halo(vol, 2, border), _expected_halo(vol, 0, 6, 2, border))
