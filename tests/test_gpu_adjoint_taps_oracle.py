"""The adjoint call with both outputs (dL/dX and all 27 tap gradients) on
f32 volumes with 9-tap passes, element-wise against the FP64 oracle.

The cases take the tensor-map loads of the input-gradient kernel (rows a
multiple of 64 long) and cover the smallest extents (9 planes, 16 rows),
ragged tile rows, several batch items, tiles touching every border, many
Z chunks, mirrored views of X and G and run-to-run repeatability.  Bounds are
relative to the stencil magnitude (the same chain on |x| and |w|): dL/dX
2e-6, tap gradients 2e-5 of their magnitude sums.
"""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import BorderMode, Image
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _taps(rng):
    out = []
    for ax in range(3):
        w = rng.standard_normal(9)
        out.append((ax, w / np.abs(w).sum()))
    return out


def _check(x, g, passes, border, gx_got, taps_got):
    """x, g: (b, z, y, x) float64 arrays as the kernel saw them."""
    apasses = [(a, np.abs(w)) for a, w in passes]
    tref, tmag = 0.0, 0.0
    for b in range(x.shape[0]):
        gref, tr = O.compose_adjoint(g[b], x[b], passes, border)
        gmag, tm = O.compose_adjoint(np.abs(g[b]), np.abs(x[b]), apasses, border)
        err = np.abs(gx_got[b].astype(np.float64) - gref)
        bad = err > 2e-6 * gmag + 1e-30
        assert not bad.any(), "dL/dX item %d: %d mismatches, worst %.3g" % (
            b, int(bad.sum()), float((err / (2e-6 * gmag + 1e-30)).max()))
        tref = tref + np.concatenate(tr)
        tmag = tmag + np.concatenate(tm)
    terr = np.abs(taps_got - tref)
    assert (terr <= 2e-5 * tmag + 1e-30).all(), float((terr / (2e-5 * tmag + 1e-30)).max())


@pytest.mark.parametrize("border", [BorderMode.Clamp, BorderMode.Reflect])
@pytest.mark.parametrize("shape", [(1, 9, 16, 64), (2, 37, 41, 128), (1, 24, 16, 192), (3, 12, 33, 64)])
def test_adjoint_with_taps_vs_oracle(border, shape):
    rng = np.random.default_rng(sum(shape) + int(border))
    x = rng.standard_normal(shape).astype(np.float32)
    g = rng.standard_normal(shape).astype(np.float32)
    passes = _taps(rng)
    xi = Image.from_tensor(torch.from_numpy(x).to(DEV))
    gi = Image.from_tensor(torch.from_numpy(g).to(DEV))
    gx = Image.empty(gi.extent(), torch.float32)
    tg = torch.zeros(27, dtype=torch.float64, device=DEV)
    n.convolve_axes_adjoint(gi, xi, gx, passes, border, tg)
    torch.cuda.synchronize()
    _check(x.astype(np.float64), g.astype(np.float64), passes, int(border), gx.tensor().cpu().numpy(),
           tg.cpu().numpy())


@pytest.mark.parametrize("border", [BorderMode.Clamp, BorderMode.Reflect])
def test_adjoint_with_taps_mirrored_views(border):
    # X and G seen through the same mirrored view (negative y and z strides)
    rng = np.random.default_rng(90 + int(border))
    shape = (2, 20, 32, 128)
    x = rng.standard_normal(shape).astype(np.float32)
    g = rng.standard_normal(shape).astype(np.float32)
    passes = _taps(rng)
    xi = Image.from_tensor(torch.from_numpy(x).to(DEV)).mirror(1).mirror(2)
    gi = Image.from_tensor(torch.from_numpy(g).to(DEV)).mirror(1).mirror(2)
    gx = Image.empty(gi.extent(), torch.float32)
    tg = torch.zeros(27, dtype=torch.float64, device=DEV)
    n.convolve_axes_adjoint(gi, xi, gx, passes, border, tg)
    torch.cuda.synchronize()
    xv = np.ascontiguousarray(x[:, ::-1, ::-1, :]).astype(np.float64)
    gv = np.ascontiguousarray(g[:, ::-1, ::-1, :]).astype(np.float64)
    _check(xv, gv, passes, int(border), gx.tensor().cpu().numpy(), tg.cpu().numpy())


def test_adjoint_with_taps_many_z_chunks():
    # many tiles per batch item: the launches split Z into chunks whose
    # boundary planes come from the neighbouring chunk's range
    rng = np.random.default_rng(7)
    shape = (1, 64, 160, 256)
    x = rng.standard_normal(shape).astype(np.float32)
    g = rng.standard_normal(shape).astype(np.float32)
    passes = _taps(rng)
    xi = Image.from_tensor(torch.from_numpy(x).to(DEV))
    gi = Image.from_tensor(torch.from_numpy(g).to(DEV))
    gx = Image.empty(gi.extent(), torch.float32)
    tg = torch.zeros(27, dtype=torch.float64, device=DEV)
    n.convolve_axes_adjoint(gi, xi, gx, passes, BorderMode.Reflect, tg)
    torch.cuda.synchronize()
    _check(x.astype(np.float64), g.astype(np.float64), passes, O.REFLECT, gx.tensor().cpu().numpy(),
           tg.cpu().numpy())


def test_adjoint_with_taps_repeatable():
    rng = np.random.default_rng(5)
    shape = (2, 30, 48, 128)
    xi = Image.from_tensor(torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(DEV))
    gi = Image.from_tensor(torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(DEV))
    passes = _taps(rng)
    outs = []
    for _ in range(2):
        gx = Image.empty(gi.extent(), torch.float32)
        tg = torch.zeros(27, dtype=torch.float64, device=DEV)
        n.convolve_axes_adjoint(gi, xi, gx, passes, BorderMode.Reflect, tg)
        outs.append((gx.tensor().clone(), tg.clone()))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
