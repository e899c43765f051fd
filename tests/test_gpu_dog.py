"""The Difference-of-Gaussians scale space of ndl::detect_keypoints
(processing/feature_detection.h:101-122) on the GPU, through the C ABI.

* 2-D images with FP32 outputs run the one-read fused kernel: its levels and
  differences are compared with the FP64 oracle (pinned to detect_keypoints
  itself in tests/test_oracle_golden.py) within 1e-6 of the stencil
  magnitude (the blur of |x| at that level; the sum of two for a
  difference).
* Other ranks and FP64 outputs run one blur per level and a difference pass;
  FP64 outputs follow the reference's exact double sequence, so they equal
  the oracle bit for bit, and the keypoints found on them equal
  detect_keypoints' own.
"""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import Image, abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-6


def blob_image(shape, nblobs, seed):
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    x = rng.random(shape) * 4.0
    for _ in range(nblobs):
        c = [rng.uniform(0, s) for s in shape]
        sg = rng.uniform(1.5, 4.0)
        x += rng.uniform(-120, 120) * np.exp(-sum((g - ci) ** 2 for g, ci in zip(grids, c)) / (2 * sg * sg))
    return x


def magnitudes(x, ns, s0):
    """Blur of |x| per level: the stencil magnitude of every output."""
    lv, _ = O.dog_scale_space(np.abs(O.to_f64(x)), ns, s0)
    return lv


def check_float(levels, dogs, x, ns, s0, code=None):
    ref_l, ref_d = O.dog_scale_space(x, ns, s0, code)
    mag = magnitudes(x if code is None else O.to_f64(x, code), ns, s0)
    for i, d in enumerate(dogs):
        err = np.abs(d.tensor().double().cpu().numpy() - ref_d[i])
        assert (err <= TOL * (mag[i] + mag[i + 1]) + 1e-30).all(), (i, float(err.max()))
    if levels is not None:
        for i, lv in enumerate(levels):
            err = np.abs(lv.tensor().double().cpu().numpy() - ref_l[i])
            assert (err <= TOL * mag[i] + 1e-30).all(), (i, float(err.max()))


@pytest.mark.parametrize("shape", [(64, 128), (200, 333), (41, 1000), (96, 50)])
def test_dog_fused_f32(shape):
    x = blob_image(shape, 30, sum(shape)).astype(np.float32)
    src = Image.from_tensor(torch.from_numpy(x).cuda())
    dogs, levels = n.dog_scale_space(src, 5, 1.6, levels=True)
    torch.cuda.synchronize()
    check_float(levels, dogs, x, 5, 1.6)


@pytest.mark.parametrize("ns,s0", [(4, 1.0), (6, 1.2), (16, 0.7)])
def test_dog_fused_scales(ns, s0):
    x = blob_image((120, 150), 30, ns).astype(np.float32)
    src = Image.from_tensor(torch.from_numpy(x).cuda())
    dogs, _ = n.dog_scale_space(src, ns, s0)
    torch.cuda.synchronize()
    check_float(None, dogs, x, ns, s0)


def test_dog_fused_u8_view():
    """uint8 source through a swapped and mirrored view; strided outputs."""
    rng = np.random.default_rng(3)
    base = rng.integers(0, 256, (150, 90), dtype=np.uint8)
    src = Image.from_tensor(torch.from_numpy(base).cuda()).swap_axes(0, 1).mirror(1)
    logical = src.tensor().cpu().numpy()
    bufs = [torch.zeros((src.extent()[0], src.extent()[1] + 3), device="cuda") for _ in range(4)]
    # ndl view ends are inclusive: extent (90, 150) of a (93, 150) buffer, then swapped
    dogs = [Image.from_tensor(b).view((0, 0), (src.extent()[1] - 1, src.extent()[0] - 1)).swap_axes(0, 1)
            for b in bufs]
    assert dogs[0].extent() == src.extent() and dogs[0].stride()[0] != 1
    n.dog_scale_space(src, 5, 1.6, dogs=dogs)
    torch.cuda.synchronize()
    check_float(None, dogs, logical, 5, 1.6)


@pytest.mark.parametrize("tdt", [torch.bfloat16, torch.float16])
def test_dog_fused_16bit_source(tdt):
    x = torch.from_numpy(blob_image((100, 140), 20, 5).astype(np.float32)).to(tdt)
    src = Image.from_tensor(x.cuda())
    dogs, _ = n.dog_scale_space(src, 5, 1.6)
    torch.cuda.synchronize()
    check_float(None, dogs, x.float().numpy(), 5, 1.6)


@pytest.mark.parametrize("shape,ns,s0", [((500,), 5, 1.6), ((24, 26, 28), 4, 0.8), ((20, 21, 22, 23), 4, 0.8)])
def test_dog_other_ranks_f32(shape, ns, s0):
    x = blob_image(shape, 10, len(shape)).astype(np.float32)
    src = Image.from_tensor(torch.from_numpy(x).cuda())
    dogs, levels = n.dog_scale_space(src, ns, s0, levels=True)
    torch.cuda.synchronize()
    check_float(levels, dogs, x, ns, s0)


@pytest.mark.parametrize("shape,ns,s0", [((64, 72), 5, 1.6), ((24, 26, 28), 4, 0.8)])
def test_dog_f64_bit_exact_and_keypoints(shape, ns, s0):
    x = blob_image(shape, 40, sum(shape))
    src = Image.from_tensor(torch.from_numpy(x).cuda())
    dogs, levels = n.dog_scale_space(src, ns, s0, levels=True, dtype=torch.float64)
    torch.cuda.synchronize()
    ref_l, ref_d = O.dog_scale_space(x, ns, s0)
    got = [d.tensor().cpu().numpy() for d in dogs]
    for i in range(ns - 1):
        assert (got[i] == ref_d[i]).all(), i
    for i in range(ns):
        assert (levels[i].tensor().cpu().numpy() == ref_l[i]).all(), i
    kp = O.dog_keypoints(got, O.dog_sigmas(ns, s0), 0.5)
    assert len(kp) >= 5
    if O.have_reference():
        assert kp == O.ref_detect_keypoints(x, ns, s0, 0.5)


def test_dog_rejects_bad_calls():
    src = Image.from_tensor(torch.zeros((40, 50), device="cuda"))
    with pytest.raises(abi.NdlGpuError) as e:
        n.dog_scale_space(src, 3, 1.6)                                   # num_scales < 4
    assert e.value.status == abi.ERR_INVALID_ARGUMENT
    small = Image.from_tensor(torch.zeros((16, 64), device="cuda"))
    with pytest.raises(abi.NdlGpuError) as e:
        n.dog_scale_space(small, 5, 1.6)                                 # radius 20 > extent 16
    assert e.value.status == abi.ERR_RADIUS_EXCEEDS_EXTENT
    d = Image.empty(src.extent(), torch.float32)
    with pytest.raises(abi.NdlGpuError) as e:
        n.dog_scale_space(src, 4, 1.0, dogs=[d, d, Image.empty(src.extent(), torch.float32)])
    assert e.value.status == abi.ERR_ALIASING
    with pytest.raises(abi.NdlGpuError) as e:
        n.dog_scale_space(src, 4, 1.0, dtype=torch.int32)
    assert e.value.status == abi.ERR_UNSUPPORTED_DTYPE
    with pytest.raises(abi.NdlGpuError) as e:
        n.dog_scale_space(src, 4, -1.0)
    assert e.value.status == abi.ERR_BAD_SIGMA


def test_dog_empty_image_is_a_no_op():
    src = Image.from_tensor(torch.zeros((0, 64), device="cuda"))
    dogs, levels = n.dog_scale_space(src, 5, 1.6, levels=True)
    assert len(dogs) == 4 and len(levels) == 5
