"""ndl::box_blur (processing/summed_area_table.h:300-339) on the GPU through
the C ABI, against the oracle restatement pinned to the compiled reference
(tests/test_oracle_golden.py): the summed-area table is built with the
reference's sequential running sums in double, so every result is compared
bit for bit, floating-point types included."""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import Image, abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(300,), (37, 41), (64, 200), (19, 23, 29), (5, 6, 7, 9)])
@pytest.mark.parametrize("radius", [1, 3, 5])
@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("dt,odt", [(np.uint8, np.uint8), (np.float32, np.float32), (np.float64, np.float64),
                                    (np.int16, np.float32)])
def test_box_blur_vs_oracle(shape, radius, border, dt, odt):
    if border != 0 and radius > min(shape):
        pytest.skip("Wrap/Reflect map one period")
    rng = np.random.default_rng(sum(shape) + radius + border)
    x = (rng.random(shape) * 200).astype(dt) if dt != np.float64 else rng.standard_normal(shape)
    src = Image.from_tensor(torch.from_numpy(x).cuda())
    dst = Image.empty(src.extent(), torch.from_numpy(np.zeros(1, odt)).dtype)
    n.box_blur(src, dst, radius, border)
    ref = O.box_blur(x, radius, border, O.dtype_code(np.zeros(1, odt)))
    assert (dst.tensor().cpu().numpy() == ref).all()


def test_box_blur_views_and_workspace():
    rng = np.random.default_rng(2)
    base = (rng.random((30, 40, 50)) * 255).astype(np.uint8)
    src = Image.from_tensor(torch.from_numpy(base).cuda()).swap_axes(0, 2).mirror(1)
    logical = src.tensor().cpu().numpy()
    buf = torch.zeros((src.extent()[2], src.extent()[1], src.extent()[0] + 5), dtype=torch.uint8, device="cuda")
    dst = Image.from_tensor(buf).view((0, 0, 0), (src.extent()[0] - 1, -1, -1))
    ws = torch.empty(64 << 20, dtype=torch.uint8, device="cuda")
    n.box_blur(src, dst, 4, 2, workspace=ws)
    assert (dst.tensor().cpu().numpy() == O.box_blur(logical, 4, 2)).all()


def test_box_blur_rejects_bad_calls():
    src = Image.from_tensor(torch.zeros((8, 10), device="cuda"))
    dst = Image.empty(src.extent(), torch.float32)
    with pytest.raises(abi.NdlGpuError):
        n.box_blur(src, dst, 0)                                          # radius must be > 0
    with pytest.raises(abi.NdlGpuError) as e:
        n.box_blur(src, dst, 9, 2)                                       # Reflect radius > extent 8
    assert e.value.status == abi.ERR_RADIUS_EXCEEDS_EXTENT
    with pytest.raises(abi.NdlGpuError) as e:
        n.box_blur(src, Image.empty([10, 9], torch.float32), 1)
    assert e.value.status == abi.ERR_EXTENT_MISMATCH
    with pytest.raises(abi.NdlGpuError) as e:
        n.box_blur(src, dst, 2, 0, workspace=torch.empty(16, dtype=torch.uint8, device="cuda"))
    assert e.value.status == abi.ERR_WORKSPACE


@pytest.mark.parametrize("dt", [np.uint8, np.float32])
def test_box_blur_clamp_radius_beyond_extent_and_empty(dt):
    """Clamp needs no period: a window wider than the image repeats the edge
    samples (the reference pads with kernelTapCoord's clamp); empty images
    are a no-op."""
    rng = np.random.default_rng(11)
    x = (rng.random((3, 40)) * 200).astype(dt)
    src = Image.from_tensor(torch.from_numpy(x).cuda())
    dst = Image.empty(src.extent(), src.dtype)
    n.box_blur(src, dst, 5, 0)
    assert (dst.tensor().cpu().numpy() == O.box_blur(x, 5, 0)).all()
    e = Image.from_tensor(torch.zeros((0, 7), dtype=torch.float32, device="cuda"))
    n.box_blur(e, Image.empty(e.extent(), torch.float32), 2, 2)
