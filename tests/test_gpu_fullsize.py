"""The hot path at the full sizes of its workloads.

The element-wise parity tests compare with the FP64 oracle at sizes it runs
in seconds.  Here every workload runs at its real shape and is checked either
against the oracle where that is still quick (the uint8 volume), or through
size-independent properties:

* configuration 2, uint8 256^3 through ``swap_axes(0,2).mirror(1)``, binomial
  taps, Wrap: bit-exact with the oracle's round-once composition;
* configuration 3, eight 192^3 f32 volumes, 9-tap Reflect chain: the adjoint
  identity <W, P X> = <P^T W, X>, and every tap gradient against the forward
  run with that tap's kernel replaced by a one-hot kernel (L is linear in each
  axis's taps, so dL/dw_a[k] = <W, P[w_a := e_k] X>);
* configuration 5, 1024x1024x3x96 BF16 and FP16 video: against the FP32 run on
  the same (decoded) values, within 4e-3 of the stencil magnitude;
* configuration 4, 512 uneven instances in one batched launch: against one
  plain FP32 call per instance (FP32 both: 1e-5 of the magnitude), and the
  BF16 batch against the FP32 plain results (4e-3).

Dot products are accumulated in FP64 on the GPU.
"""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import BorderMode, Image, abi
from ndl_b200.batch import Batch
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda"


def dot64(a, b):
    return float((a.double() * b.double()).sum())


def test_config2_u8_full_view_bit_exact():
    rng = np.random.default_rng(20)
    base = rng.integers(0, 256, (256, 256, 256), dtype=np.uint8)
    src = Image.from_tensor(torch.from_numpy(base).to(DEV)).swap_axes(0, 2).mirror(1)
    assert src.stride()[1] < 0
    w = np.array([1, 4, 6, 4, 1]) / 16.0
    passes = [(0, w), (1, w), (2, w)]
    dst = Image.empty(src.extent(), torch.uint8)
    n.convolve_axes(src, dst, passes, BorderMode.Wrap, compose=abi.ROUND_ONCE)
    logical = src.tensor().cpu().numpy()
    ref = O.compose(logical, passes, O.WRAP, O.U8)
    assert (dst.tensor().cpu().numpy() == ref).all()


def _config3(seed=30):
    g = torch.Generator(device=DEV)
    g.manual_seed(seed)
    shape = (8, 192, 192, 192)
    X = torch.randn(shape, generator=g, device=DEV)
    W = torch.randn(shape, generator=g, device=DEV)
    rng = np.random.default_rng(seed)
    passes = []
    for ax in range(3):
        w = rng.standard_normal(9)
        passes.append((ax, w / np.abs(w).sum()))
    return X, W, passes


def test_config3_full_adjoint_identity_and_tap_gradients():
    X, W, passes = _config3()
    xi, wi = Image.from_tensor(X), Image.from_tensor(W)
    Y = torch.empty_like(X)
    n.convolve_axes(xi, Image.from_tensor(Y), passes, BorderMode.Reflect)
    GX = torch.empty_like(X)
    taps = torch.zeros(27, dtype=torch.float64, device=DEV)
    n.convolve_axes_adjoint(wi, xi, Image.from_tensor(GX), passes, BorderMode.Reflect, taps)
    torch.cuda.synchronize()
    # <W, P X> = <P^T W, X>
    lhs, rhs = dot64(W, Y), dot64(GX, X)
    scale = float((W.double() * Y.double()).abs().sum() + (GX.double() * X.double()).abs().sum())
    assert abs(lhs - rhs) <= 1e-6 * scale, (lhs, rhs, scale)
    # dL/dw_a[k] = <W, P[w_a := e_k] X> for a spread of taps on every axis
    Yk = torch.empty_like(X)
    got = taps.cpu().numpy()
    for a in range(3):
        for k in (0, 3, 4, 8):
            pk = [(ax, (np.eye(9)[k] if ax == a else w)) for ax, w in passes]
            n.convolve_axes(xi, Image.from_tensor(Yk), pk, BorderMode.Reflect)
            ref = dot64(W, Yk)
            mag = float((W.double() * Yk.double()).abs().sum())
            assert abs(got[9 * a + k] - ref) <= 1e-5 * mag, (a, k, got[9 * a + k], ref, mag)


@pytest.mark.parametrize("tdt", [torch.bfloat16, torch.float16])
def test_config5_video_full_16bit_vs_f32(tdt):
    g = torch.Generator(device=DEV)
    g.manual_seed(50)
    shape = (96, 3, 1024, 1024)       # (t, c, y, x): ndl axes x, y, c, t
    v = torch.rand(shape, generator=g, device=DEV)
    salt = torch.rand(shape, generator=g, device=DEV) < 0.01
    v = torch.where(salt, torch.ones_like(v), v).to(tdt)
    vf = v.float()
    sig = (2.5, 2.5, 0.0, 1.5)
    passes = [(ax, O.gaussian_weights(s)) for ax, s in enumerate(sig) if s > 0]
    out16 = Image.empty(Image.from_tensor(v).extent(), tdt)
    out32 = Image.empty(Image.from_tensor(vf).extent(), torch.float32)
    n.convolve_axes(Image.from_tensor(v), out16, passes, BorderMode.Reflect)
    n.convolve_axes(Image.from_tensor(vf), out32, passes, BorderMode.Reflect)
    # inputs in [0, 1] and positive normalised taps: the stencil magnitude is
    # the output itself
    err = (out16.tensor().float() - out32.tensor()).abs()
    assert float((err - 4e-3 * out32.tensor().abs()).max()) <= 0.0, float((err / out32.tensor().abs().clamp_min(1e-30)).max())
    # adjoint of the same chain
    g16 = Image.empty(Image.from_tensor(v).extent(), tdt)
    g32 = Image.empty(Image.from_tensor(vf).extent(), torch.float32)
    n.convolve_axes_adjoint(Image.from_tensor(v), None, g16, passes, BorderMode.Reflect)
    n.convolve_axes_adjoint(Image.from_tensor(vf), None, g32, passes, BorderMode.Reflect)
    err = (g16.tensor().float() - g32.tensor()).abs()
    assert float((err - 4e-3 * g32.tensor().abs()).max()) <= 0.0


def test_config4_full_batch_vs_plain_calls():
    import bench
    inst = bench.config4_instances()
    g = torch.Generator(device=DEV)
    g.manual_seed(40)
    xs = [torch.rand(sh, generator=g, device=DEV) for sh, _, _ in inst]
    b32, b16 = Batch(), Batch()
    out32, out16, x16 = [], [], []
    for (sh, passes, border), x in zip(inst, xs):
        o = Image.empty(Image.from_tensor(x).extent(), torch.float32)
        b32.add(Image.from_tensor(x), o, passes, border)
        out32.append(o)
        xb = x.to(torch.bfloat16)
        ob = Image.empty(Image.from_tensor(xb).extent(), torch.bfloat16)
        b16.add(Image.from_tensor(xb), ob, passes, border)
        out16.append(ob)
        x16.append(xb)
    b32.plan()
    b16.plan()
    b32.launch()
    b16.launch()
    torch.cuda.synchronize()
    for (sh, passes, border), x, xb, o32, o16 in zip(inst, xs, x16, out32, out16):
        ref = Image.empty(Image.from_tensor(x).extent(), torch.float32)
        n.convolve_axes(Image.from_tensor(x), ref, passes, border)
        r = ref.tensor()
        # inputs in [0, 1), positive Gaussian taps: the magnitude is the output
        assert float(((o32.tensor() - r).abs() - 1e-5 * r.abs()).max()) <= 1e-30, (sh, border)
        refb = Image.empty(Image.from_tensor(xb).extent(), torch.float32)
        n.convolve_axes(Image.from_tensor(xb.float()), refb, passes, border)
        rb = refb.tensor()
        assert float(((o16.tensor().float() - rb).abs() - 4e-3 * rb.abs()).max()) <= 1e-30, (sh, border)
    b32.close()
    b16.close()
