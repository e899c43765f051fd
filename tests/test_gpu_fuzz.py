"""Seeded random cases over the fused widths: random extents (ragged tiles,
axes shorter than a tile), a random view of the source (axis swaps and
mirrors), every border, f32 / bf16 / f16 storage, the forward of random
positive taps, and the input and tap gradients of random taps, each against the FP64 oracle on the same (decoded) values.  The
tolerances are the ones of the other parity tests: 1e-6 of the stencil
magnitude for f32 results, 4e-3 for 16-bit storage, and for the tap
gradients 2e-5 of the largest one."""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import Image
from oracle import oracle as O

pytestmark = pytest.mark.gpu

WIDTHS_VOL = [3, 5, 7, 9, 11, 13]
WIDTHS_IMG = [3, 5, 7, 9, 11, 13, 15, 17]


def _view(rng, img, nswap):
    """A random view of img: a swap among its first nswap axes (the ones the
    passes run along), and mirrors of any axis."""
    v = img
    d = len(v.extent())
    if nswap >= 2 and rng.random() < 0.5:
        a, b = rng.choice(nswap, 2, replace=False)
        v = v.swap_axes(int(a), int(b))
    for a in range(d):
        if rng.random() < 0.3:
            v = v.mirror(a)
    return v


def _case(seed):
    rng = np.random.default_rng(1000 + seed)
    vol = rng.random() < 0.5
    k = int(rng.choice(WIDTHS_VOL if vol else WIDTHS_IMG))
    lo = k // 2 + 1
    if vol:
        shape = tuple(int(s) for s in rng.integers(max(lo, 5), 40, size=3))
    else:
        shape = (int(rng.integers(1, 4)),) + tuple(int(s) for s in rng.integers(max(lo, 5), 90, size=2))
    border = int(rng.integers(0, 3))
    return rng, vol, k, shape, border


@pytest.mark.parametrize("seed", range(40))
def test_fuzz_forward(seed):
    rng, vol, k, shape, border = _case(seed)
    tdt = [torch.float32, torch.bfloat16, torch.float16][int(rng.integers(0, 3))]
    x = torch.from_numpy(rng.random(shape).astype(np.float32) + 0.1).to(tdt)
    src = _view(rng, Image.from_tensor(x.cuda()), 3 if vol else 2)
    logical = src.tensor().float().cpu().numpy().astype(np.float64)
    npass = 3 if vol else 2
    passes = [(a, rng.random(k) + 0.05) for a in range(npass)]      # positive taps: magnitude = result
    out = Image.empty(src.extent(), tdt)
    n.convolve_axes(src, out, passes, border)
    ref = O.compose_total(logical, passes, border)
    got = out.tensor().float().cpu().numpy().astype(np.float64)
    tol = 1e-6 if tdt == torch.float32 else 4e-3
    assert (np.abs(got - ref) <= tol * np.abs(ref) + 1e-30).all(), (seed, vol, k, shape, border, tdt)


@pytest.mark.parametrize("seed", range(40))
def test_fuzz_gradients(seed):
    rng, vol, k, shape, border = _case(seed)
    npass = 3 if vol else 2
    x = rng.standard_normal(shape).astype(np.float32)
    g = rng.standard_normal(shape).astype(np.float32)
    passes = [(a, rng.standard_normal(k)) for a in range(npass)]
    xi = _view(rng, Image.from_tensor(torch.from_numpy(x).cuda()), npass)
    xl = xi.tensor().cpu().numpy().astype(np.float64)
    gt = torch.from_numpy(rng.standard_normal(xl.shape).astype(np.float32))
    gi = Image.from_tensor(gt.cuda())
    gx = Image.empty(gi.extent(), torch.float32)
    taps = torch.zeros(npass * k, dtype=torch.float64, device="cuda")
    n.convolve_axes_adjoint(gi, xi, gx, passes, border, taps)
    gl = gt.numpy().astype(np.float64)
    # batch axes (the image case's leading axis) are independent
    if vol:
        ref_gx, ref_t = O.compose_adjoint(gl, xl, passes, border)
        ref_t = np.concatenate(ref_t)
    else:
        parts = [O.compose_adjoint(gl[b], xl[b], passes, border) for b in range(xl.shape[0])]
        ref_gx = np.stack([p[0] for p in parts])
        ref_t = np.sum([np.concatenate(p[1]) for p in parts], axis=0)
    got = gx.tensor().cpu().numpy().astype(np.float64)
    mag = np.abs(gl)
    for a, w in passes[::-1]:
        if vol:
            mag = O.axis_pass_adjoint(mag, a, np.abs(w), border)
    if not vol:
        mag = np.stack([_adj_mag(np.abs(gl[b]), passes, border) for b in range(gl.shape[0])])
    assert (np.abs(got - ref_gx) <= 1e-6 * mag + 1e-30).all(), (seed, vol, k, shape, border)
    t = taps.cpu().numpy()
    assert np.abs(t - ref_t).max() <= 2e-5 * np.abs(ref_t).max(), (seed, vol, k, shape, border)


def _adj_mag(gabs, passes, border):
    m = gabs
    for a, w in passes[::-1]:
        m = O.axis_pass_adjoint(m, a, np.abs(w), border)
    return m
