"""The tiled per-axis pass kernels (any width, FP32 sums, float storage)
against the FP64 oracle.

They run the plain path's passes where no fused kernel is compiled: Gaussians
wider than the fused widths (volumes above 19 taps, images above 25), uneven
per-axis widths, four-axis chains, strided and mirrored views, 16-bit
storage, and more outer lines than a launch grid's second dimension holds.  Bounds are relative to the stencil magnitude (the same chain on
|x| and |w|): FP32 1e-6; 16-bit storage 4e-3 (FP32 intermediates, one
rounding at the end).
"""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import BorderMode, Image, abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"
BORDERS = [BorderMode.Clamp, BorderMode.Wrap, BorderMode.Reflect]


def _check(got, x, passes, border, tol):
    ref = O.compose_total(x.astype(np.float64), passes, int(border))
    mag = O.compose_total(np.abs(x).astype(np.float64), [(a, np.abs(w)) for a, w in passes], int(border))
    err = np.abs(got.astype(np.float64) - ref)
    bound = tol * mag + 1e-30
    assert (err <= bound).all(), float((err / bound).max())


@pytest.mark.parametrize("border", BORDERS)
@pytest.mark.parametrize("sigma", [3.4, 4.0, 6.0])
@pytest.mark.parametrize("shape", [(40, 48, 72), (21, 33, 150)])
def test_wide_gaussian_volume(border, sigma, shape):
    rng = np.random.default_rng(int(10 * sigma) + int(border) + shape[0])
    x = rng.standard_normal(shape).astype(np.float32)
    s = Image.from_tensor(torch.from_numpy(x).to(DEV))
    o = Image.empty(s.extent(), torch.float32)
    n.gaussian_blur(s, o, sigma, border)
    w = O.gaussian_weights(sigma)
    _check(o.tensor().cpu().numpy(), x, [(a, w) for a in range(3)], border, 1e-6)


@pytest.mark.parametrize("border", BORDERS)
@pytest.mark.parametrize("sigma", [4.5, 8.0])
def test_wide_gaussian_image(border, sigma):
    rng = np.random.default_rng(int(10 * sigma) + int(border))
    x = rng.standard_normal((300, 257)).astype(np.float32)
    s = Image.from_tensor(torch.from_numpy(x).to(DEV))
    o = Image.empty(s.extent(), torch.float32)
    n.gaussian_blur(s, o, sigma, border)
    w = O.gaussian_weights(sigma)
    _check(o.tensor().cpu().numpy(), x, [(0, w), (1, w)], border, 1e-6)


@pytest.mark.parametrize("border", BORDERS)
def test_uneven_widths_random_taps(border):
    # 5, 21 and 3 taps (no fused kernel for the combination), asymmetric taps
    rng = np.random.default_rng(70 + int(border))
    x = rng.standard_normal((24, 70, 96)).astype(np.float32)
    passes = []
    for ax, k in ((0, 5), (1, 21), (2, 3)):
        w = rng.standard_normal(k)
        passes.append((ax, w / np.abs(w).sum()))
    s = Image.from_tensor(torch.from_numpy(x).to(DEV))
    o = Image.empty(s.extent(), torch.float32)
    before = int(abi.load().ndlgpu_kernel_launches())
    n.convolve_axes(s, o, passes, border)
    torch.cuda.synchronize()
    assert int(abi.load().ndlgpu_kernel_launches()) - before == 3
    _check(o.tensor().cpu().numpy(), x, passes, border, 1e-6)


@pytest.mark.parametrize("border", BORDERS)
def test_four_axis_chain_and_views(border):
    # four passes on a 4-D view with a mirrored and a swapped axis
    rng = np.random.default_rng(80 + int(border))
    base = rng.standard_normal((6, 10, 40, 64)).astype(np.float32)
    s = Image.from_tensor(torch.from_numpy(base).to(DEV)).mirror(1).swap_axes(2, 3)
    logical = s.tensor().cpu().numpy()
    passes = []
    for ax, k in ((0, 23), (1, 7), (2, 3), (3, 5)):
        w = rng.random(k) + 0.1
        passes.append((ax, w / w.sum()))
    o = Image.empty(s.extent(), torch.float32)
    n.convolve_axes(s, o, passes, border)
    _check(o.tensor().cpu().numpy(), logical, passes, border, 1e-6)


@pytest.mark.parametrize("tdt", [torch.bfloat16, torch.float16])
def test_wide_gaussian_16bit_storage(tdt):
    rng = np.random.default_rng(90)
    x = rng.random((36, 40, 130)).astype(np.float32)
    s = Image.from_tensor(torch.from_numpy(x).to(DEV).to(tdt))
    o = Image.empty(s.extent(), tdt)
    n.gaussian_blur(s, o, 5.0, BorderMode.Reflect)
    xd = s.tensor().float().cpu().numpy()
    w = O.gaussian_weights(5.0)
    # FP32 intermediates, one rounding to 16 bits at the end
    _check(o.tensor().float().cpu().numpy(), xd, [(a, w) for a in range(3)], BorderMode.Reflect, 4e-3)


@pytest.mark.parametrize("border", [BorderMode.Clamp, BorderMode.Reflect])
def test_strided_pass_many_outer_lines(border):
    # a pass along an axis of extent 2 whose outer index (the other axes but
    # x) runs past 65535 lines, and odd row counts for the x pass: the
    # persistent tile walk's index decomposition
    rng = np.random.default_rng(100 + int(border))
    x = rng.standard_normal((300, 301, 2, 33)).astype(np.float32)     # (w, z, y, x)
    passes = []
    for ax, k in ((0, 5), (1, 3), (2, 7), (3, 3)):
        w = rng.standard_normal(k)
        passes.append((ax, w / np.abs(w).sum()))
    s = Image.from_tensor(torch.from_numpy(x).to(DEV))
    o = Image.empty(s.extent(), torch.float32)
    n.convolve_axes(s, o, passes, border)
    _check(o.tensor().cpu().numpy(), x, passes, border, 1e-6)
