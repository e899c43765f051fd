"""The packed uint8 forward (two 16-bit lanes per word, one 32-bit multiply-
add per word and tap) against the oracle, bit for bit.

It serves uint8 volumes with non-negative dyadic taps whose Y and X-of-Y
sums of bytes stay below 2^16 ([1,4,6,4,1]/16 and [1,2,1]/4 per axis), with
one rounding at the end (round-once composition) or a single pass.  Cases:
every border mode, ragged extents in all three axes, several batch items, a
plain layout and views whose destination is contiguous along another axis
(swap_axes / mirror), and the launch route (one launch of the packed kernel).
"""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import BorderMode, Image, abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"
BINOMIAL = np.array([1, 4, 6, 4, 1]) / 16.0
TENT = np.array([1, 2, 1]) / 4.0


def _run(base, view, w, border):
    src = view(Image.from_tensor(torch.from_numpy(base).to(DEV)))
    dst = Image.empty(src.extent(), torch.uint8)
    passes = [(0, w), (1, w), (2, w)]
    n.convolve_axes(src, dst, passes, border, compose=abi.ROUND_ONCE)
    logical = src.tensor().cpu().numpy()
    ref = O.compose(logical, passes, int(border), O.U8)
    return dst.tensor().cpu().numpy(), ref


@pytest.mark.parametrize("border", [BorderMode.Clamp, BorderMode.Wrap, BorderMode.Reflect])
@pytest.mark.parametrize("w", [BINOMIAL, TENT], ids=["binomial", "tent"])
@pytest.mark.parametrize("shape", [(40, 48, 64), (33, 50, 80), (9, 31, 144), (7, 20, 100)])
def test_u8_plain_layout_bit_exact(border, w, shape):
    rng = np.random.default_rng(sum(shape) + int(border) + len(w))
    base = rng.integers(0, 256, shape, dtype=np.uint8)
    got, ref = _run(base, lambda im: im, w, border)
    assert (got == ref).all(), int((got != ref).sum())


@pytest.mark.parametrize("border", [BorderMode.Clamp, BorderMode.Wrap, BorderMode.Reflect])
@pytest.mark.parametrize("shape", [(64, 64, 64), (70, 37, 48)])
def test_u8_transposed_view_bit_exact(border, shape):
    # the workload's view: the destination is contiguous along the source's
    # slowest axis, and one axis is mirrored
    rng = np.random.default_rng(3 * sum(shape) + int(border))
    base = rng.integers(0, 256, shape, dtype=np.uint8)
    got, ref = _run(base, lambda im: im.swap_axes(0, 2).mirror(1), BINOMIAL, border)
    assert (got == ref).all(), int((got != ref).sum())


def test_u8_batch_items_bit_exact():
    rng = np.random.default_rng(11)
    base = rng.integers(0, 256, (3, 20, 40, 64), dtype=np.uint8)     # (b, z, y, x)
    src = Image.from_tensor(torch.from_numpy(base).to(DEV))
    dst = Image.empty(src.extent(), torch.uint8)
    passes = [(0, BINOMIAL), (1, BINOMIAL), (2, BINOMIAL)]
    n.convolve_axes(src, dst, passes, BorderMode.Wrap, compose=abi.ROUND_ONCE)
    got = dst.tensor().cpu().numpy()
    for b in range(3):
        ref = O.compose(base[b], passes, O.WRAP, O.U8)
        assert (got[b] == ref).all()


def test_u8_takes_the_packed_kernel():
    rng = np.random.default_rng(12)
    base = rng.integers(0, 256, (32, 32, 64), dtype=np.uint8)
    src = Image.from_tensor(torch.from_numpy(base).to(DEV))
    dst = Image.empty(src.extent(), torch.uint8)
    passes = [(0, TENT), (1, TENT), (2, TENT)]
    before = int(abi.load().ndlgpu_kernel_launches())
    n.convolve_axes(src, dst, passes, BorderMode.Reflect, compose=abi.ROUND_ONCE)
    torch.cuda.synchronize()
    assert int(abi.load().ndlgpu_kernel_launches()) - before == 1
    ref = O.compose(base, passes, O.REFLECT, O.U8)
    assert (dst.tensor().cpu().numpy() == ref).all()
