"""Gradcheck harness of the adjoint (the C ABI behind torch.autograd).

* torch.autograd.gradcheck on FP64 tensors for every border mode (our FP64
  kernels; finite differences against the analytic adjoint).
* config 3: a 192^3 FP64 volume, per-axis 9-tap N(0,1) kernels normalised
  to unit L1 norm, Reflect, L = sum(W * Y): dL/dX at 64 random coordinates
  and all 27 tap gradients against FP64 central differences with step 1e-3,
  and the whole gradient against the FP64 oracle's (oracle/ndl_oracle.c).
* the FP32 kernels against the same FP64 oracle gradient.
"""
import numpy as np
import pytest
import torch

from ndl_b200 import abi
from ndl_b200.autograd import separable_conv
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def l1_taps(rng, k):
    w = rng.standard_normal(k)
    return w / np.abs(w).sum()


@pytest.mark.parametrize("border", [abi.CLAMP, abi.WRAP, abi.REFLECT])
def test_torch_gradcheck_fp64(border):
    rng = np.random.default_rng(border)
    x = torch.tensor(rng.standard_normal((5, 6, 7)), dtype=torch.float64, device="cuda", requires_grad=True)
    taps = [torch.tensor(l1_taps(rng, k), dtype=torch.float64, device="cuda", requires_grad=True) for k in (5, 3, 5)]
    fn = lambda x_, a, b, c: separable_conv(x_, [a, b, c], [0, 1, 2], border)
    assert torch.autograd.gradcheck(fn, (x, *taps), eps=1e-6, atol=1e-8, rtol=1e-6)


def test_config3_fd_and_oracle_gradient():
    rng = np.random.default_rng(20261203)
    N = 192
    xn = rng.standard_normal((N, N, N))
    wn = rng.standard_normal((N, N, N))
    tn = [l1_taps(rng, 9) for _ in range(3)]
    x = torch.tensor(xn, device="cuda", requires_grad=True)
    W = torch.tensor(wn, device="cuda")
    taps = [torch.tensor(t, device="cuda", requires_grad=True) for t in tn]
    border = abi.REFLECT

    def loss(x_, tp):
        return (W * separable_conv(x_, tp, [0, 1, 2], border)).sum()

    L = loss(x, taps)
    L.backward()
    gx = x.grad.detach().cpu().numpy()
    gtap = [t.grad.detach().cpu().numpy() for t in taps]

    # FP64 oracle gradient (the literal transpose, oracle/ndl_oracle.c)
    passes = [(a, tn[a]) for a in range(3)]
    gx_ref, tap_ref = O.compose_adjoint(wn, xn, passes, O.REFLECT)
    assert np.abs(gx - gx_ref).max() <= 1e-12 * np.abs(gx_ref).max()
    for a in range(3):
        assert np.abs(gtap[a] - tap_ref[a]).max() <= 1e-10 * np.abs(tap_ref[a]).max()

    # central finite differences, step 1e-3.  L is linear in x and in each
    # tap vector, so the quotient is exact up to rounding; the two forward
    # results are subtracted before the sum against W to keep that rounding
    # small.
    h = 1e-3
    coords = rng.integers(0, N, size=(64, 3))
    with torch.no_grad():
        def fwd(x_, tp):
            return separable_conv(x_, tp, [0, 1, 2], border)
        for (i, j, k) in coords:
            xp = x.detach().clone()
            xp[i, j, k] += h
            yp = fwd(xp, taps)
            xp[i, j, k] -= 2 * h
            ym = fwd(xp, taps)
            fd = ((W * (yp - ym)).sum() / (2 * h)).item()
            assert abs(fd - gx[i, j, k]) <= 1e-7 * max(1.0, abs(gx[i, j, k])), (i, j, k, fd, gx[i, j, k])
        for a in range(3):
            for k in range(9):
                tp = [t.detach().clone() for t in taps]
                tp[a][k] += h
                yp = fwd(x.detach(), tp)
                tp[a][k] -= 2 * h
                ym = fwd(x.detach(), tp)
                fd = ((W * (yp - ym)).sum() / (2 * h)).item()
                assert abs(fd - gtap[a][k]) <= 1e-7 * max(1.0, abs(gtap[a][k])), (a, k, fd, gtap[a][k])


@pytest.mark.parametrize("border", [abi.CLAMP, abi.WRAP, abi.REFLECT])
def test_fp32_gradients_vs_fp64_oracle(border):
    rng = np.random.default_rng(100 + border)
    shape = (40, 48, 56)
    xn = rng.standard_normal(shape).astype(np.float32)
    wn = rng.standard_normal(shape).astype(np.float32)
    tn = [l1_taps(rng, 9).astype(np.float32) for _ in range(3)]
    x = torch.tensor(xn, device="cuda", requires_grad=True)
    W = torch.tensor(wn, device="cuda")
    taps = [torch.tensor(t, device="cuda", requires_grad=True) for t in tn]
    (W * separable_conv(x, taps, [0, 1, 2], border)).sum().backward()
    gx_ref, tap_ref = O.compose_adjoint(wn, xn, [(a, tn[a].astype(np.float64)) for a in range(3)], border)
    err = np.abs(x.grad.cpu().numpy() - gx_ref).max() / np.abs(gx_ref).max()
    assert err <= 2e-6, err
    for a in range(3):
        terr = np.abs(taps[a].grad.cpu().numpy() - tap_ref[a]).max() / np.abs(tap_ref[a]).max()
        assert terr <= 2e-5, (a, terr)
