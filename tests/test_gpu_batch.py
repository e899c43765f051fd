"""The batched form against the FP64 oracle: uneven 2-D and 3-D instances
with per-axis tap counts up to 37, mixed borders, forward and adjoint, in one
persistent launch; every compiled tile shape; graph replay; BF16 storage."""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import Image, abi
from ndl_b200.batch import Batch, tile_configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make_instances(rng, count, dtype=torch.float32, max_sigma=6.0):
    inst = []
    for i in range(count):
        three = (i % 2 == 1)
        if three:
            shape = tuple(int(v) for v in np.exp(rng.uniform(np.log(10), np.log(40), 3)))
        else:
            shape = tuple(int(v) for v in np.exp(rng.uniform(np.log(16), np.log(200), 2)))
        border = int(rng.integers(0, 3))
        passes = []
        for ax in range(len(shape)):
            extent = shape[::-1][ax]
            sig = float(rng.uniform(0.5, max_sigma))
            while border != 0 and O.gaussian_radius(sig) > extent:
                sig *= 0.5
            passes.append((ax, O.gaussian_weights(sig)))
        x = rng.random(shape).astype(np.float32)
        adjoint = bool(rng.integers(0, 2))
        inst.append((x, passes, border, adjoint))
    return inst


def oracle_out(x, passes, border, adjoint, code=None):
    xd = O.to_f64(x, code)
    if not adjoint:
        return O.compose_total(xd, passes, border)
    g = xd
    for ax, w in passes[::-1]:
        g = O.axis_pass_adjoint(g, ax, w, border)
    return g


def magnitude(x, passes, border, adjoint, code=None):
    return oracle_out(np.abs(O.to_f64(x, code)), [(a, np.abs(w)) for a, w in passes], border, adjoint)


@pytest.mark.parametrize("cfg", range(4))
def test_batch_f32_all_tile_configs(cfg):
    rng = np.random.default_rng(100 + cfg)
    inst = make_instances(rng, 14)
    b = Batch()
    outs = []
    for x, passes, border, adj in inst:
        src = Image.from_tensor(torch.from_numpy(x).cuda())
        dst = Image.empty(src.extent(), torch.float32)
        b.add(src, dst, passes, border, adjoint=adj)
        outs.append(dst)
    try:
        b.plan(cfg)
    except abi.NdlGpuError:
        pytest.skip("tile configuration does not fit the widest taps")
    b.launch()
    torch.cuda.synchronize()
    for (x, passes, border, adj), dst in zip(inst, outs):
        ref = oracle_out(x, passes, border, adj)
        mag = magnitude(x, passes, border, adj)
        err = np.abs(dst.tensor().cpu().numpy() - ref)
        assert (err <= 1e-6 * mag + 1e-30).all(), (x.shape, border, adj, (err / (mag + 1e-30)).max())


def test_batch_graph_replay_and_bf16():
    rng = np.random.default_rng(7)
    inst = make_instances(rng, 10, max_sigma=3.0)
    b = Batch()
    outs = []
    ins = []
    for x, passes, border, adj in inst:
        t = torch.from_numpy(x).cuda().to(torch.bfloat16)
        src = Image.from_tensor(t)
        dst = Image.empty(src.extent(), torch.bfloat16)
        b.add(src, dst, passes, border, adjoint=adj)
        outs.append(dst)
        ins.append(src)
    b.plan()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.graph_launch(s)
        b.graph_launch(s)
    s.synchronize()
    first = [o.tensor().clone() for o in outs]
    with torch.cuda.stream(s):
        b.graph_launch(s)
    s.synchronize()
    for a, o in zip(first, outs):
        assert torch.equal(a, o.tensor())
    for (x, passes, border, adj), src, dst in zip(inst, ins, outs):
        xb = src.tensor().contiguous().view(torch.int16).cpu().numpy().view(np.uint16)
        ref = oracle_out(xb, passes, border, adj, O.BF16)
        mag = magnitude(xb, passes, border, adj, O.BF16)
        got = O.to_f64(dst.tensor().contiguous().view(torch.int16).cpu().numpy().view(np.uint16), O.BF16)
        err = np.abs(got - ref)
        assert (err <= 4e-3 * mag + 1e-30).all(), (x.shape, border, adj, (err / (mag + 1e-30)).max())


def test_batch_autotune_picks_a_fitting_config(tmp_path, monkeypatch):
    from ndl_b200 import autotune
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tiles.json"))
    rng = np.random.default_rng(3)
    inst = make_instances(rng, 6)
    b = Batch()
    for x, passes, border, adj in inst:
        src = Image.from_tensor(torch.from_numpy(x).cuda())
        b.add(src, Image.empty(src.extent(), torch.float32), passes, border, adjoint=adj)
    cfg, times = autotune.best_tile_config(b, iters=2)
    assert cfg in range(len(tile_configs())) and times
    cfg2, _ = autotune.best_tile_config(b)     # from the cache
    assert cfg2 == cfg
