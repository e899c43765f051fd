"""ndl::gradient (processing/convolution.h:359-388) on the GPU, through the C
ABI, against the FP64 oracle restatement pinned to the compiled reference
(tests/test_oracle_golden.py).  The central difference (x[i+1] - x[i-1]) / 2
is exact in FP32 up to one final rounding, the same single rounding the
reference's double accumulation and cast make, so every result is compared
bit for bit."""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import BorderMode, Image, abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def ndl_dst(src, dtype):
    """dst of extent {DIM, ...src}: the component axis is ndl axis 0 (the
    last torch dim), as ndl's default layout puts it."""
    return Image.empty([src.dim] + src.extent(), dtype)


@pytest.mark.parametrize("shape", [(300,), (37, 41), (40, 64), (19, 23, 29), (16, 24, 32), (4, 64, 64, 64)])
@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("dt,odt", [(np.float32, np.float32), (np.uint8, np.int16), (np.int32, np.int32),
                                    (np.float64, np.float64), (np.uint8, np.float32)])
def test_gradient_vs_oracle(shape, border, dt, odt):
    rng = np.random.default_rng(sum(shape) + border)
    x = rng.standard_normal(shape).astype(dt) if dt in (np.float32, np.float64) else (rng.random(shape) * 250).astype(dt)
    src = Image.from_tensor(torch.from_numpy(x).cuda())
    dst = ndl_dst(src, torch.from_numpy(np.zeros(1, odt)).dtype)
    n.gradient(src, dst, border)
    ref = O.gradient(x, border, O.dtype_code(np.zeros(1, odt)))
    assert (dst.tensor().cpu().numpy() == ref).all()


def test_gradient_views_and_default_border():
    rng = np.random.default_rng(9)
    base = rng.standard_normal((20, 30, 40)).astype(np.float32)
    src = Image.from_tensor(torch.from_numpy(base).cuda()).swap_axes(0, 2).mirror(1)
    logical = src.tensor().cpu().numpy()
    # the component axis slowest in memory: a swapped view of a {x, y, z, DIM} buffer
    buf = torch.zeros((3,) + logical.shape, device="cuda")          # torch (DIM, z', y', x')
    dst = Image.from_tensor(buf)                                     # ndl extent (x', y', z', DIM)
    # move the component axis (ndl 3) to the front: swap 0<->3, then restore the order of the rest
    dst = dst.swap_axes(0, 3).swap_axes(1, 3).swap_axes(2, 3)
    assert dst.extent() == [3] + src.extent()
    n.gradient(src, dst)                                             # default: Reflect
    ref = O.gradient(logical, O.REFLECT)
    assert (dst.tensor().cpu().numpy() == ref).all()


def test_gradient_rejects_bad_destinations():
    src = Image.from_tensor(torch.zeros((8, 9), device="cuda"))
    with pytest.raises(abi.NdlGpuError):
        n.gradient(src, Image.empty([3, 9, 8], torch.float32))       # leading extent != DIM
    with pytest.raises(abi.NdlGpuError):
        n.gradient(src, Image.empty([9, 8], torch.float32))          # no component axis
    with pytest.raises(abi.NdlGpuError):
        n.gradient(src, Image.empty([2, 9, 7], torch.float32))       # extents differ
