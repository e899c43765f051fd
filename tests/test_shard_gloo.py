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
