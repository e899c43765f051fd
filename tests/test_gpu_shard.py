"""One volume split into slabs along its slowest axis (ndl_b200.shard): each
rank's blur of its halo-extended slab equals, plane for plane, the blur of
the whole volume.  The ranks are two processes sharing this GPU and trading
halos through gloo on the host (no kernel waits on another rank); on a
multi-GPU node the same code moves the halos with NCCL."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

SIG = (2.5, 2.5, 0.0, 1.5)     # x, y, -, t (ndl axis order): r_t = 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _volume(dt):
    g = torch.Generator().manual_seed(5)
    v = torch.rand((24, 3, 64, 96), generator=g)                 # (t, c, y, x)
    return v.to(dt)


def _worker(rank, world, port, dt, border, q):
    import torch.distributed as dist
    from ndl_b200.shard import sharded_gaussian_blur_axes, slab_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        vol = _volume(dt)
        a, b = slab_bounds(vol.shape[0], world, rank)
        out = sharded_gaussian_blur_axes(vol[a:b].contiguous().cuda(), SIG, border)
        torch.cuda.synchronize()
        # by value (numpy): a shared-memory tensor could outlive this process
        q.put((rank, a, b, out.cpu().float().numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dt", [torch.float32, torch.bfloat16])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_slabs_equal_whole_volume(dt, border):
    import ndl_b200 as n
    from ndl_b200 import Image
    vol = _volume(dt).cuda()
    whole = Image.empty(Image.from_tensor(vol).extent(), dt)
    n.gaussian_blur_axes(Image.from_tensor(vol), whole, list(SIG), border)
    ref = whole.tensor().cpu()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, 2, port, dt, border, q)) for k in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, a, b, out in res:
        assert torch.equal(torch.from_numpy(out), ref[a:b].float()), (rank, border)


def test_single_rank_slab_is_the_whole_blur():
    import ndl_b200 as n
    from ndl_b200 import Image
    from ndl_b200.shard import sharded_gaussian_blur_axes
    vol = _volume(torch.float32).cuda()
    whole = Image.empty(Image.from_tensor(vol).extent(), torch.float32)
    n.gaussian_blur_axes(Image.from_tensor(vol), whole, list(SIG), 2)
    assert torch.equal(sharded_gaussian_blur_axes(vol, SIG, 2), whole.tensor())
