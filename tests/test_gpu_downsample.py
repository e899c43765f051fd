"""ndl::downsample (processing/convolution.h:241-305) on the GPU through the
C ABI, against the oracle restatement pinned to the compiled reference
(tests/test_oracle_golden.py): the block sums run in double in the
reference's order, so every result is compared bit for bit."""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import Image, abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _data(shape, dt, rng):
    if np.issubdtype(dt, np.integer):
        return (rng.random(shape) * 250 - (120 if dt not in (np.uint8,) else 0)).astype(dt)
    return rng.standard_normal(shape).astype(dt)


@pytest.mark.parametrize("shape,factor,ch", [((30, 40, 3), 2, 0), ((31, 17, 3), 3, 0), ((9, 10, 11), 4, 1),
                                             ((5, 7, 9, 2), 2, 3), ((33, 21), 5, 1), ((6, 50), 7, 0),
                                             ((720, 1280, 3), 2, 0), ((3, 720, 1280), 8, 2)])
@pytest.mark.parametrize("dt", [np.uint8, np.int16, np.int32, np.float32, np.float64])
def test_downsample_vs_oracle(shape, factor, ch, dt):
    rng = np.random.default_rng(sum(shape) + factor)
    x = _data(shape, dt, rng)
    out = n.downsample(Image.from_tensor(torch.from_numpy(x).cuda()), factor, ch)
    ref = O.downsample(x, factor, ch)
    got = out.tensor().cpu().numpy()
    assert got.shape == ref.shape and (got == ref).all()


def test_downsample_views_and_other_dst_type():
    rng = np.random.default_rng(4)
    base = rng.integers(0, 256, (40, 3, 64), dtype=np.uint8)
    src = Image.from_tensor(torch.from_numpy(base).cuda()).swap_axes(1, 2).mirror(0)   # ndl {64, 40, 3} view
    logical = src.tensor().cpu().numpy()
    out = n.downsample(src, 3, 2)
    assert (out.tensor().cpu().numpy() == O.downsample(logical, 3, 2)).all()
    # float dst of a uint8 source: the average itself (no rounding)
    ext = out.extent()
    f = n.downsample(src, 3, 2, dst=Image.empty(ext, torch.float32))
    assert (f.tensor().cpu().numpy() == O.downsample(logical, 3, 2, out_code=O.F32)).all()


def test_downsample_rejects_bad_calls():
    src = Image.from_tensor(torch.zeros((8, 10, 3), device="cuda"))
    with pytest.raises(abi.NdlGpuError):
        n.downsample(src, 1, 0)                                         # factor must be > 1
    with pytest.raises(abi.NdlGpuError) as e:
        n.downsample(src, 2, 0, dst=Image.empty([3, 4, 4], torch.float32))
    assert e.value.status == abi.ERR_EXTENT_MISMATCH
    with pytest.raises(abi.NdlGpuError):
        n.downsample(src, 2, 5)                                         # channel axis out of range
    with pytest.raises(abi.NdlGpuError):
        n.downsample(Image.from_tensor(torch.zeros(16, device="cuda")), 2, 0)   # rank 1


@pytest.mark.parametrize("shape,ch", [((300, 400, 3), 0), ((3, 170, 290), 2), ((400, 3), 0), ((12, 33, 34, 2), 0)])
@pytest.mark.parametrize("dt", [np.uint8, np.float32])
def test_per_channel_blur(shape, ch, dt):
    """ndl::per_channel(src, dst, channelAxis, gaussian_blur(., ., 1.3, b))
    is gaussian_blur_axes with sigma 0 on the channel axis: bit-exact for
    uint8 (exact integer path), within 1e-6 of the stencil magnitude for
    f32 (FP32 accumulation; inputs and taps are positive)."""
    rng = np.random.default_rng(sum(shape))
    x = (rng.random(shape) * 200).astype(dt)
    src = Image.from_tensor(torch.from_numpy(x).cuda())
    sig = [0.0 if a == ch else 1.3 for a in range(len(shape))]
    for b in (0, 1, 2):
        dst = Image.empty(src.extent(), src.dtype)
        n.gaussian_blur_axes(src, dst, sig, b)
        ref = O.per_channel_blur(x, 1.3, ch, b)
        got = dst.tensor().cpu().numpy()
        if dt == np.uint8:
            assert (got == ref).all(), b
        else:
            assert (np.abs(got.astype(np.float64) - ref) <= 1e-6 * np.abs(ref) + 1e-30).all(), b


def test_downsample_factor_beyond_extent_and_empty():
    """A factor larger than an axis leaves one output averaging the whole
    axis; an empty source is a no-op."""
    rng = np.random.default_rng(12)
    x = (rng.random((4, 3, 2)) * 255).astype(np.uint8)          # ndl {2, 3, 4}, channel axis 0
    out = n.downsample(Image.from_tensor(torch.from_numpy(x).cuda()), 5, 0)
    assert out.extent() == [2, 1, 1]
    assert (out.tensor().cpu().numpy() == O.downsample(x, 5, 0)).all()
    e = Image.from_tensor(torch.zeros((0, 6, 3), dtype=torch.uint8, device="cuda"))
    n.downsample(e, 2, 0)
