"""Parity of the sm_100a kernels (through the C ABI) with the reference.

Checks against (a) golden fixtures the compiled reference produced
(tests/golden, made by make_golden.py) and (b) the FP64 oracle on seeded
inputs, over every border mode, element type, view layout and the edge cases
the reference's tests touch (tiny and ragged extents, extent-1 axes, empty
images, negative strides).

Tolerances: integral results bit-exact; FP64 and EXACT-precision results
bit-exact; FP32 results within 1e-6 of the reference relative to the
magnitude of the stencil sum, |gpu - ref| <= 1e-6 * (|w| * |x|)(i), which is
the plain 1e-6 relative error wherever data and weights are positive;
bf16/f16 storage within 4e-3 relative to that same magnitude.
"""
import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import BorderMode, Image, abi
from oracle import oracle as O
from conftest import golden

pytestmark = pytest.mark.gpu

DEV = "cuda"


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def host(t):
    t = t.detach()
    if t.dtype == torch.bfloat16:
        return t.contiguous().view(torch.int16).cpu().numpy().view(np.uint16)
    return t.cpu().numpy()


def magnitude(x, passes, border):
    """(|w| * |x|): the stencil sum of absolute values, per output."""
    ax = np.abs(O.to_f64(x))
    return O.compose_total(ax, [(a, np.abs(np.asarray(w, np.float64))) for a, w in passes], border)


def assert_close(got, ref, mag, tol, what=""):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    err = np.abs(got - ref)
    bound = tol * mag + 1e-30
    bad = err > bound
    assert not bad.any(), "%s: %d mismatches, worst err %.3g vs bound %.3g" % (
        what, bad.sum(), (err / bound).max(), bound.flat[np.argmax(err / bound)])


# ---------------------------------------------------------------------------
# Golden fixtures from the compiled reference
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("sigma", [2.0, 1.3])
def test_golden_gaussian_f32(border, sigma):
    d, _ = golden("gauss2d_f32")
    src = d["src"]
    s = Image.from_tensor(dev(src))
    o = Image.empty(s.extent(), torch.float32)
    n.gaussian_blur(s, o, sigma, border)
    ref = d["out_b%d_s%s" % (border, str(sigma).replace(".", "p"))]
    w = O.gaussian_weights(sigma)
    assert_close(host(o.tensor()), ref, magnitude(src, [(0, w), (1, w)], border), 1e-6, "gaussian f32")


@pytest.mark.parametrize("border", [0, 1, 2])
def test_golden_gaussian_u8_exact(border):
    # non-dyadic weights: the reference's double sequence, bit-exact
    d, _ = golden("u8_gauss_s1p5")
    s = Image.from_tensor(dev(d["src"]))
    o = Image.empty(s.extent(), torch.uint8)
    n.gaussian_blur(s, o, 1.5, border)
    assert (host(o.tensor()) == d["out_b%d" % border]).all()


@pytest.mark.parametrize("dst_layout", ["contiguous", "same_view"])
def test_golden_u8_binomial_view(dst_layout):
    d, _ = golden("u8_binomial_view")
    base = dev(d["base"])
    src = Image.from_tensor(base).swap_axes(0, 2).mirror(1)
    assert src.stride()[1] < 0
    w = d["taps"]
    passes = [(0, w), (1, w), (2, w)]
    for mode, key in ((abi.ROUND_ONCE, "round_once"), (abi.CAST_EACH, "cast_each")):
        if dst_layout == "contiguous":
            dst = Image.empty(src.extent(), torch.uint8)
        else:
            dst = Image.from_tensor(torch.zeros_like(base)).swap_axes(0, 2).mirror(1)
        n.convolve_axes(src, dst, passes, BorderMode.Wrap, compose=mode)
        assert (host(dst.tensor()) == d[key]).all(), key


def test_golden_unit_known_answers():
    d, _ = golden("unit_known_answers")
    img = Image.from_tensor(dev(d["img"]))
    for b in (0, 1, 2):
        for kk, key in ((np.ones((3, 3), np.int32), "sum3_b%d" % b), (np.ones((5, 5), np.int32), "sum5_b%d" % b)):
            out = Image.zeros(img.extent(), torch.int32)
            n.convolve(img, out, kk, b)
            assert (host(out.tensor()) == d[key]).all(), key
    i54 = Image.from_tensor(dev(d["img54"]))
    out = Image.zeros(i54.extent(), torch.int32)
    n.convolve(i54, out, d["kb"], BorderMode.Wrap)
    assert (host(out.tensor()) == d["composite_wrap"]).all()
    assert host(out.tensor()).sum() == d["kb"].sum() * d["img54"].sum()
    f = Image.from_tensor(dev(d["fimg"]))
    out = Image.zeros(f.extent(), torch.float64)
    n.convolve(f, out, d["fk"], BorderMode.Wrap)
    assert (host(out.tensor()) == d["fft_wrap"]).all()     # FP64: bit-exact


def test_golden_one_d():
    d, _ = golden("one_d")
    a = Image.from_tensor(dev(d["a"]))
    out = Image.zeros(a.extent(), torch.float32)
    n.convolve(a, out, d["box"], BorderMode.Clamp)
    got = host(out.tensor())
    # EXPECT_FLOAT_EQ in type_coverage_tests.cpp:148 (4 ulps)
    assert abs(float(got[1]) - (3.0 + 5.0 + 7.0) / 3.0) <= 4 * np.spacing(np.float32(5.0))
    assert np.allclose(got, d["out_box"], rtol=1e-6, atol=0)
    x6 = Image.from_tensor(dev(d["x6"]))
    o6 = Image.zeros(x6.extent(), torch.uint8)
    n.gaussian_blur(x6, o6, 2.0, BorderMode.Reflect)      # DIM == 1: truncating convolve()
    assert (host(o6.tensor()) == d["out_g1"]).all()


def test_golden_rand9_reflect_fused():
    d, _ = golden("f32_rand9_reflect")
    t = d["taps"]
    passes = [(0, t[0]), (1, t[1]), (2, t[2])]
    s = Image.from_tensor(dev(d["src"]))
    o = Image.empty(s.extent(), torch.float32)
    n.convolve_axes(s, o, passes, BorderMode.Reflect)
    assert_close(host(o.tensor()), d["out_f64"], magnitude(d["src"], passes, 2), 1e-6, "rand9")
    # EXACT precision reproduces the reference's float result bit for bit
    o2 = Image.empty(s.extent(), torch.float32)
    n.convolve_axes(s, o2, passes, BorderMode.Reflect, precision=abi.PREC_EXACT)
    assert (host(o2.tensor()) == d["out"]).all()


def test_golden_video4d():
    d, _ = golden("video4d_f32")
    s = Image.from_tensor(dev(d["src"]))
    o = Image.empty(s.extent(), torch.float32)
    n.gaussian_blur_axes(s, o, [2.5, 2.5, 0.0, 1.5], BorderMode.Reflect)
    gx, gt = O.gaussian_weights(2.5), O.gaussian_weights(1.5)
    mag = magnitude(d["src"], [(0, gx), (1, gx), (3, gt)], 2)
    assert_close(host(o.tensor()), d["out_f64"], mag, 1e-6, "video f32")
    for tdt, tol in ((torch.bfloat16, 4e-3), (torch.float16, 4e-3)):
        sb = Image.from_tensor(dev(d["src"]).to(tdt))
        ob = Image.empty(s.extent(), tdt)
        n.gaussian_blur_axes(sb, ob, [2.5, 2.5, 0.0, 1.5], BorderMode.Reflect)
        xin = host(sb.tensor())
        code = O.BF16 if tdt == torch.bfloat16 else O.F16
        ref = O.compose_total(O.to_f64(xin, code), [(0, gx), (1, gx), (3, gt)], 2)
        got = O.to_f64(host(ob.tensor()), code)
        assert_close(got, ref, mag, tol, str(tdt))


def test_golden_u8_trunc_axis():
    d, _ = golden("u8_trunc_axis")
    s = Image.from_tensor(dev(d["src"]))
    for ax in range(3):
        kshape = [1, 1, 1]
        kshape[2 - ax] = 5
        o = Image.zeros(s.extent(), torch.uint8)
        n.convolve(s, o, d["taps"].reshape(kshape), BorderMode.Reflect)
        assert (host(o.tensor()) == d["ax%d" % ax]).all(), ax


# ---------------------------------------------------------------------------
# Seeded cases against the FP64 oracle
# ---------------------------------------------------------------------------

def rand_array(rng, shape, dt):
    if dt in (np.uint8,):
        return rng.integers(0, 256, shape).astype(dt)
    if dt in (np.int16,):
        return rng.integers(-300, 300, shape).astype(dt)
    if dt in (np.int32,):
        return rng.integers(-100000, 100000, shape).astype(dt)
    return rng.standard_normal(shape).astype(dt)


SHAPES_3D = [(1, 1, 1), (5, 3, 2), (9, 13, 17), (33, 70, 65), (40, 31, 130), (3, 97, 5)]


@pytest.mark.parametrize("shape", SHAPES_3D)
@pytest.mark.parametrize("border", [0, 1, 2])
def test_f32_three_axes_vs_oracle(shape, border):
    rng = np.random.default_rng(hash((shape, border)) % 2**32)
    x = rand_array(rng, shape, np.float32)
    passes = []
    for ax in range(3):
        K = 2 * min(4, shape[2 - ax]) + 1 if border != 0 else 9
        w = rng.standard_normal(K)
        passes.append((ax, w / np.abs(w).sum()))
    s = Image.from_tensor(dev(x))
    o = Image.empty(s.extent(), torch.float32)
    n.convolve_axes(s, o, passes, border)
    ref = O.compose_total(x, passes, border)
    assert_close(host(o.tensor()), ref, magnitude(x, passes, border), 1e-6, "f32 3-axis %s" % (shape,))
    # the EXACT path is the reference's own sequence, bit for bit
    o2 = Image.empty(s.extent(), torch.float32)
    n.convolve_axes(s, o2, passes, border, precision=abi.PREC_EXACT)
    assert (host(o2.tensor()) == O.cast(ref, O.F32)).all()


@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("mode", [abi.ROUND_ONCE, abi.CAST_EACH])
def test_u8_binomial_vs_oracle_ragged(border, mode):
    rng = np.random.default_rng(border * 7 + mode)
    for shape in [(3, 5, 7), (17, 64, 33), (70, 9, 129)]:
        x = rand_array(rng, shape, np.uint8)
        w = np.array([1, 4, 6, 4, 1]) / 16.0
        passes = [(0, w), (1, w), (2, w)]
        s = Image.from_tensor(dev(x))
        o = Image.empty(s.extent(), torch.uint8)
        n.convolve_axes(s, o, passes, border, compose=mode)
        ref = O.compose(x, passes, border, O.U8, O.STORE_ROUND if mode == abi.ROUND_ONCE else O.STORE_CAST)
        assert (host(o.tensor()) == ref).all(), shape


@pytest.mark.parametrize("dt", [np.uint8, np.int16, np.int32, np.float64])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_exact_types_gaussian(dt, border):
    rng = np.random.default_rng(11)
    x = rand_array(rng, (21, 30), dt)
    s = Image.from_tensor(dev(x))
    o = Image.zeros(s.extent(), torch.from_numpy(x).dtype)
    n.gaussian_blur(s, o, 1.7, border)
    ref = O.gaussian_blur(x, 1.7, border)
    assert (host(o.tensor()) == ref).all()


@pytest.mark.parametrize("ops", [
    [("mirror", 0)],
    [("swap", 0, 1)],
    [("swap", 0, 2), ("mirror", 1)],
    [("view", 0, 1, -2, 2)],
    [("view", 1, 0, -1, -3), ("swap", 1, 2)],
])
@pytest.mark.parametrize("dt", [np.float32, np.uint8])
def test_views_vs_oracle(ops, dt):
    rng = np.random.default_rng(3)
    base = rand_array(rng, (12, 23, 40), dt)
    t = dev(base)
    src = Image.from_tensor(t)
    npv = base
    for op in ops:
        if op[0] == "swap":
            src = src.swap_axes(op[1], op[2])
            a, b = npv.ndim - 1 - op[1], npv.ndim - 1 - op[2]
            npv = np.swapaxes(npv, a, b)
        elif op[0] == "mirror":
            src = src.mirror(op[1])
            npv = np.flip(npv, npv.ndim - 1 - op[1])
        else:
            _, ax, s0, e0, st = op
            start = [0, 0, 0]
            end = [-1, -1, -1]
            step = [1, 1, 1]
            start[ax], end[ax], step[ax] = s0, e0, st
            src = src.view(start, end, step)
            na = npv.ndim - 1 - ax
            L = npv.shape[na]
            s1 = s0 % L if s0 < 0 else s0
            e1 = e0 % L if e0 < 0 else e0
            sl = [slice(None)] * npv.ndim
            sl[na] = slice(s1, e1 + 1, st) if st > 0 else slice(e1, s1 - 1 if s1 > 0 else None, st)
            npv = npv[tuple(sl)]
    assert list(src.tensor().shape) == list(npv.shape)
    assert (host(src.tensor()) == npv).all()
    w = np.array([1, 4, 6, 4, 1]) / 16.0 if dt == np.uint8 else np.array([0.2, -0.1, 0.5, 0.3, 0.1])
    passes = [(0, w), (1, w), (2, w)]
    for border in (0, 1, 2):
        o = Image.empty(src.extent(), torch.from_numpy(base).dtype)
        n.convolve_axes(src, o, passes, border)
        if dt == np.uint8:
            assert (host(o.tensor()) == O.compose(npv, passes, border, O.U8)).all()
        else:
            assert_close(host(o.tensor()), O.compose_total(npv, passes, border), magnitude(npv, passes, border),
                         1e-6, "view")


def test_extent_one_axes_and_single_tap():
    rng = np.random.default_rng(1)
    x = rand_array(rng, (1, 7, 1), np.float32)
    s = Image.from_tensor(dev(x))
    for border in (0, 1, 2):
        passes = [(0, [0.25, 0.5, 0.25]), (1, [0.3, 0.4, 0.3]), (2, [1.0])]
        o = Image.empty(s.extent(), torch.float32)
        n.convolve_axes(s, o, passes, border)
        ref = O.compose_total(x, passes, border)
        assert_close(host(o.tensor()), ref, magnitude(x, passes, border), 1e-6, "extent-1")


def test_empty_image():
    s = Image.empty([0, 4], torch.float32)
    o = Image.empty([0, 4], torch.float32)
    n.gaussian_blur(s, o, 1.0)
    torch.cuda.synchronize()


def test_nd_kernel_float_and_zero_taps():
    rng = np.random.default_rng(2)
    x = rand_array(rng, (19, 26), np.float32)
    k = rng.standard_normal((3, 5))
    k[1, 2] = 0.0
    s = Image.from_tensor(dev(x))
    for border in (0, 1, 2):
        o = Image.empty(s.extent(), torch.float32)
        n.convolve(s, o, k, border)
        ref = O.convolve_total(x, k, border)
        mag = O.convolve_total(np.abs(x), np.abs(k), border)
        assert_close(host(o.tensor()), ref, mag, 1e-6, "nd")
        o2 = Image.empty(s.extent(), torch.float32)
        n.convolve(s, o2, k, border, precision=abi.PREC_EXACT)
        assert (host(o2.tensor()) == O.cast(ref, O.F32)).all()


def test_workspace_given_by_caller():
    rng = np.random.default_rng(4)
    x = rand_array(rng, (20, 30, 40), np.float64)
    s = Image.from_tensor(dev(x))
    o = Image.empty(s.extent(), torch.float64)
    w = [0.1, 0.2, 0.4, 0.2, 0.1]
    passes = [(0, w), (1, w), (2, w)]
    nb = n.convolve_axes_workspace_size(s, o, passes)
    assert nb >= 2 * x.size * 8
    ws = torch.empty(nb, dtype=torch.uint8, device=DEV)
    n.convolve_axes(s, o, passes, workspace=ws)
    assert (host(o.tensor()) == O.compose_total(x, passes, 0)).all()


# ---------------------------------------------------------------------------
# Adjoint
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_adjoint_vs_fp64_oracle(border, dt):
    rng = np.random.default_rng(17 + border)
    shape = (11, 14, 17)
    x = rand_array(rng, shape, dt)
    g = rand_array(rng, shape, dt)
    passes = []
    for ax in range(3):
        w = rng.standard_normal(9 if border == 0 or ax > 0 else 7)
        passes.append((ax, w / np.abs(w).sum()))
    gx_ref, taps_ref = O.compose_adjoint(g, x, passes, border)
    tg = torch.zeros(sum(len(w) for _, w in passes), dtype=torch.float64, device=DEV)
    gxi = Image.empty(list(shape[::-1]), torch.from_numpy(x).dtype)
    n.convolve_axes_adjoint(Image.from_tensor(dev(g)), Image.from_tensor(dev(x)), gxi, passes, border, tg)
    got = host(gxi.tensor()).astype(np.float64)
    tol = 1e-12 if dt == np.float64 else 2e-6
    scale = np.abs(gx_ref).max()
    assert np.abs(got - gx_ref).max() <= tol * scale * 10
    tref = np.concatenate(taps_ref)
    tscale = np.abs(tref).max()
    assert np.abs(host(tg) - tref).max() <= tol * tscale * 100


@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("shape", [(9, 10, 11), (20, 33, 70), (64, 48, 130), (5, 200, 66)])
def test_fused_adjoint_input_gradient(border, shape):
    """dL/dX alone runs the fused transposed kernel (zone tables at the
    borders); checked against the FP64 oracle's literal transpose."""
    rng = np.random.default_rng(sum(shape) + border)
    g = rand_array(rng, shape, np.float32)
    passes = []
    for ax in range(3):
        w = rng.standard_normal(9)
        passes.append((ax, w / np.abs(w).sum()))
    if border != 0 and min(shape) < 4:
        pytest.skip("radius exceeds extent")
    gxi = Image.empty(list(shape[::-1]), torch.float32)
    n.convolve_axes_adjoint(Image.from_tensor(dev(g)), None, gxi, passes, border, None)
    gcur = g.astype(np.float64)
    for ax, w in passes[::-1]:
        gcur = O.axis_pass_adjoint(gcur, ax, w, border)
    mag = np.abs(g.astype(np.float64))
    for ax, w in passes[::-1]:
        mag = O.axis_pass_adjoint(mag, ax, np.abs(w), border)
    assert_close(host(gxi.tensor()), gcur, mag, 1e-6, "fused adjoint %s" % (shape,))


@pytest.mark.parametrize("tdt", [torch.float32, torch.bfloat16, torch.float16])
def test_fused_adjoint_video(tdt):
    rng = np.random.default_rng(9)
    x = rng.random((7, 3, 40, 70)).astype(np.float32)
    gx_, gt_ = O.gaussian_weights(2.5), O.gaussian_weights(1.5)
    passes = [(0, gx_), (1, gx_), (3, gt_)]
    gi = Image.from_tensor(dev(x).to(tdt))
    out = Image.empty(gi.extent(), tdt)
    n.convolve_axes_adjoint(gi, None, out, passes, BorderMode.Reflect, None)
    code = {torch.float32: O.F32, torch.bfloat16: O.BF16, torch.float16: O.F16}[tdt]
    gin = O.to_f64(host(gi.tensor()), code)
    ref = gin
    for ax, w in passes[::-1]:
        ref = O.axis_pass_adjoint(ref, ax, w, 2)
    got = O.to_f64(host(out.tensor()), code)
    tol = 1e-6 if tdt == torch.float32 else 4e-3
    mag = np.abs(gin)
    for ax, w in passes[::-1]:
        mag = O.axis_pass_adjoint(mag, ax, np.abs(w), 2)
    assert_close(got, ref, mag, tol, "video adjoint %s" % tdt)


@pytest.mark.parametrize("border", [0, 1, 2])
def test_fused_tap_gradients_views_and_batch(border):
    """Tap gradients through the fused kernel: X seen through a mirrored,
    axis-swapped view, a batch axis left untouched, every tap reported in the
    caller's tap order."""
    rng = np.random.default_rng(31 + border)
    base = rng.standard_normal((3, 30, 41, 70)).astype(np.float32)     # (b, z, y, x)
    g = rng.standard_normal((3, 30, 41, 70)).astype(np.float32)
    taps = [rng.standard_normal(9) for _ in range(3)]
    xt = dev(base)
    xi = Image.from_tensor(xt).mirror(0).mirror(2)                       # negative strides on x and z
    npx = base[:, ::-1, :, ::-1]
    passes = [(0, taps[0]), (1, taps[1]), (2, taps[2])]
    tg = torch.zeros(27, dtype=torch.float64, device=DEV)
    gi = Image.from_tensor(dev(g))
    gx = Image.empty(gi.extent(), torch.float32)
    n.convolve_axes_adjoint(gi, xi, gx, passes, border, tg)
    ref_gx, ref_t = [], []
    for b in range(3):
        a, t = O.compose_adjoint(g[b].astype(np.float64), np.ascontiguousarray(npx[b]).astype(np.float64), passes,
                                 border)
        ref_gx.append(a)
        ref_t.append(np.concatenate(t))
    tref = np.sum(ref_t, axis=0)
    got = host(tg)
    assert np.abs(got - tref).max() <= 2e-5 * np.abs(tref).max(), np.abs(got - tref).max() / np.abs(tref).max()
    gref = np.stack(ref_gx)
    assert np.abs(host(gx.tensor()) - gref).max() <= 2e-6 * np.abs(gref).max()


@pytest.mark.parametrize("tdt", [torch.bfloat16, torch.float16])
def test_fused_tap_gradients_video_16bit(tdt):
    rng = np.random.default_rng(77)
    x = rng.random((12, 2, 40, 72)).astype(np.float32)
    g = rng.standard_normal((12, 2, 40, 72)).astype(np.float32)
    gx_, gt_ = O.gaussian_weights(2.5), O.gaussian_weights(1.5)
    passes = [(0, gx_), (1, gx_), (3, gt_)]
    xi = Image.from_tensor(dev(x).to(tdt))
    gi = Image.from_tensor(dev(g).to(tdt))
    tg = torch.zeros(17 + 17 + 11, dtype=torch.float32, device=DEV)
    n.convolve_axes_adjoint(gi, xi, None, passes, BorderMode.Reflect, tg)
    code = O.BF16 if tdt == torch.bfloat16 else O.F16
    xd = O.to_f64(host(xi.tensor()), code)
    gd = O.to_f64(host(gi.tensor()), code)
    _, tref = O.compose_adjoint(gd, xd, passes, 2)
    tref = np.concatenate(tref)
    got = host(tg).astype(np.float64)
    assert np.abs(got - tref).max() <= 1e-4 * np.abs(tref).max()


@pytest.mark.parametrize("sigma", [0.5, 1.0, 1.5, 2.0, 2.3, 2.5, 3.0])
@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("shape", [(40, 48, 72), (3, 19, 23, 29)])
def test_gaussian_blur_volume_fused_sigmas(sigma, border, shape):
    """gaussian_blur of volumes at sigma 0.5 .. 3 (5, 7, 11, 13, 15, 17 and
    19 taps), the fused 3-pass kernels for those widths, within 1e-6 of the
    FP64 oracle (positive data and taps: the magnitude is the result)."""
    rng = np.random.default_rng(int(sigma * 10) + border)
    x = rng.random(shape).astype(np.float32)
    s = Image.from_tensor(torch.from_numpy(x).cuda())
    o = Image.empty(s.extent(), torch.float32)
    if len(shape) == 4:
        sig = [sigma, sigma, sigma, 0.0]
        n.gaussian_blur_axes(s, o, sig, border)
        w = O.gaussian_weights(sigma)
        ref = O.compose_total(x, [(a, w) for a in range(3)], border)
    else:
        n.gaussian_blur(s, o, sigma, border)
        ref = O.gaussian_blur(x, sigma, border, O.F64)
    got = o.tensor().cpu().numpy().astype(np.float64)
    assert (np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-30).all()


@pytest.mark.parametrize("sigma", [0.5, 1.0, 1.2, 1.5, 2.3, 2.5, 3.0, 3.3, 3.6, 4.0])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_gaussian_blur_image_fused_sigmas(sigma, border):
    """gaussian_blur of 2-D f32 images at every width from 5 to 25 taps (the
    fused 2-pass kernels), on a ragged image and on a transposed, mirrored
    view, within 1e-6 of the FP64 oracle."""
    rng = np.random.default_rng(int(sigma * 10) + 7 * border)
    x = rng.random((300, 333)).astype(np.float32)
    base = Image.from_tensor(torch.from_numpy(x).cuda())
    for s in (base, base.swap_axes(0, 1).mirror(0)):
        logical = s.tensor().cpu().numpy()
        o = Image.empty(s.extent(), torch.float32)
        n.gaussian_blur(s, o, sigma, border)
        ref = O.gaussian_blur(logical, sigma, border, O.F64)
        got = o.tensor().cpu().numpy().astype(np.float64)
        assert (np.abs(got - ref) <= 1e-6 * np.abs(ref) + 1e-30).all()


@pytest.mark.parametrize("k", [3, 5, 7, 9, 11, 13])
@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("shape", [(21, 34, 70), (2, 45, 67)])
def test_small_filter_forward_and_input_gradient(k, border, shape):
    """Small learnable filters: forward and dL/dX of k taps per axis on
    volumes (3 passes) and on batches of 2-D images (2 passes; the leading
    axis untouched), the fused kernels, against the FP64 oracle."""
    rng = np.random.default_rng(k + 10 * border + len(shape))
    two_d = shape[0] == 2
    if not two_d and k == 9:
        pytest.skip("9x9x9 is covered by the configuration-3 tests")
    x = rand_array(rng, shape, np.float32)
    g = rand_array(rng, shape, np.float32)
    axes = (0, 1) if two_d else (0, 1, 2)
    passes = []
    for ax in axes:
        w = rng.standard_normal(k)
        passes.append((ax, w / np.abs(w).sum()))
    y = Image.empty(list(shape[::-1]), torch.float32)
    n.convolve_axes(Image.from_tensor(dev(x)), y, passes, border)
    ref = O.compose_total(x, passes, border)
    mag = O.compose_total(np.abs(x.astype(np.float64)), [(a, np.abs(w)) for a, w in passes], border)
    assert_close(host(y.tensor()), ref, mag, 1e-6, "forward k=%d %s" % (k, shape))
    gxi = Image.empty(list(shape[::-1]), torch.float32)
    n.convolve_axes_adjoint(Image.from_tensor(dev(g)), None, gxi, passes, border, None)
    gcur = g.astype(np.float64)
    gmag = np.abs(gcur)
    for ax, w in passes[::-1]:
        gcur = O.axis_pass_adjoint(gcur, ax, w, border)
        gmag = O.axis_pass_adjoint(gmag, ax, np.abs(w), border)
    assert_close(host(gxi.tensor()), gcur, gmag, 1e-6, "adjoint k=%d %s" % (k, shape))


@pytest.mark.parametrize("tdt", [torch.bfloat16, torch.float16])
@pytest.mark.parametrize("shape,sigmas", [((40, 48, 72), (0.5, 1.0, 1.5, 2.0)),
                                          ((150, 170), (0.5, 1.2, 2.3, 3.0, 3.6, 4.0))])
def test_gaussian_blur_16bit_fused_widths(tdt, shape, sigmas):
    """BF16/FP16 storage with FP32 accumulation at the fused widths of
    volumes and images: within 4e-3 of the FP64 oracle run on the same
    decoded values (positive data: the magnitude is the result)."""
    rng = np.random.default_rng(len(shape))
    x = torch.from_numpy(rng.random(shape).astype(np.float32)).to(tdt)
    decoded = x.float().numpy().astype(np.float64)
    s = Image.from_tensor(x.cuda())
    for sigma in sigmas:
        for border in (0, 1, 2):
            o = Image.empty(s.extent(), tdt)
            n.gaussian_blur(s, o, sigma, border)
            ref = O.gaussian_blur(decoded, sigma, border, O.F64)
            got = o.tensor().float().cpu().numpy().astype(np.float64)
            assert (np.abs(got - ref) <= 4e-3 * np.abs(ref) + 1e-30).all(), (sigma, border)


@pytest.mark.parametrize("k", [3, 5, 7, 11, 13])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_small_filter_tap_gradients(k, border):
    """All 3k tap gradients of a k-tap-per-axis filter on a batch of volumes
    (one fused pass over X and G; the window starts off the 16-byte grid),
    through mirrored views, against the FP64 oracle's literal transpose."""
    rng = np.random.default_rng(77 + 3 * k + border)
    base = rng.standard_normal((2, 23, 37, 70)).astype(np.float32)      # (b, z, y, x)
    g = rng.standard_normal((2, 23, 37, 70)).astype(np.float32)
    taps = [rng.standard_normal(k) for _ in range(3)]
    xi = Image.from_tensor(dev(base)).mirror(0).mirror(2)
    npx = base[:, ::-1, :, ::-1]
    passes = [(0, taps[0]), (1, taps[1]), (2, taps[2])]
    tg = torch.zeros(3 * k, dtype=torch.float64, device=DEV)
    gi = Image.from_tensor(dev(g))
    gx = Image.empty(gi.extent(), torch.float32)
    n.convolve_axes_adjoint(gi, xi, gx, passes, border, tg)
    ref_gx, ref_t = [], []
    for b in range(2):
        a, t = O.compose_adjoint(g[b].astype(np.float64), np.ascontiguousarray(npx[b]).astype(np.float64), passes,
                                 border)
        ref_gx.append(a)
        ref_t.append(np.concatenate(t))
    tref = np.sum(ref_t, axis=0)
    got = host(tg)
    assert np.abs(got - tref).max() <= 2e-5 * np.abs(tref).max(), np.abs(got - tref).max() / np.abs(tref).max()
    gref = np.stack(ref_gx)
    assert np.abs(host(gx.tensor()) - gref).max() <= 2e-6 * np.abs(gref).max()


@pytest.mark.parametrize("border", [0, 1, 2])
def test_general_adjoint_two_passes(border):
    """The general (non-fused) input and tap gradients of a two-pass chain:
    a zero tap keeps the chain off the fused kernels, and two passes use one
    intermediate buffer."""
    rng = np.random.default_rng(90 + border)
    shape = (3, 37, 52)                                  # a batch of 2-D images
    x = rand_array(rng, shape, np.float32)
    g = rand_array(rng, shape, np.float32)
    w0 = rng.standard_normal(7)
    w0[2] = 0.0
    w1 = rng.standard_normal(5)
    passes = [(0, w0), (1, w1)]
    tg = torch.zeros(12, dtype=torch.float64, device=DEV)
    gxi = Image.empty(list(shape[::-1]), torch.float32)
    n.convolve_axes_adjoint(Image.from_tensor(dev(g)), Image.from_tensor(dev(x)), gxi, passes, border, tg)
    gx_only = Image.empty(list(shape[::-1]), torch.float32)
    n.convolve_axes_adjoint(Image.from_tensor(dev(g)), None, gx_only, passes, border, None)
    ref_gx, ref_t = [], []
    for b in range(3):
        a, t = O.compose_adjoint(g[b].astype(np.float64), x[b].astype(np.float64), passes, border)
        ref_gx.append(a)
        ref_t.append(np.concatenate(t))
    gref = np.stack(ref_gx)
    tref = np.sum(ref_t, axis=0)
    for got in (host(gxi.tensor()), host(gx_only.tensor())):
        assert np.abs(got - gref).max() <= 2e-6 * np.abs(gref).max()
    assert np.abs(host(tg) - tref).max() <= 2e-5 * np.abs(tref).max()


@pytest.mark.parametrize("k", [3, 5, 9, 13])
@pytest.mark.parametrize("border", [0, 1, 2])
@pytest.mark.parametrize("shape", [(3, 45, 70), (61, 83)])
def test_image_filter_tap_gradients(k, border, shape):
    """Tap gradients of a two-pass (image) filter through the fused kernel:
    a batch of images streamed as planes, and a single image, with dL/dX in
    the same call; against the FP64 oracle's literal transpose."""
    rng = np.random.default_rng(300 + k + 5 * border + len(shape))
    x = rng.standard_normal(shape).astype(np.float32)
    g = rng.standard_normal(shape).astype(np.float32)
    taps = [rng.standard_normal(k) for _ in range(2)]
    passes = [(0, taps[0]), (1, taps[1])]
    tg = torch.zeros(2 * k, dtype=torch.float64, device=DEV)
    gi = Image.from_tensor(dev(g))
    gx = Image.empty(gi.extent(), torch.float32)
    n.convolve_axes_adjoint(gi, Image.from_tensor(dev(x)), gx, passes, border, tg)
    xs = x if len(shape) == 3 else x[None]
    gs = g if len(shape) == 3 else g[None]
    ref_gx, ref_t = [], []
    for b in range(xs.shape[0]):
        a, t = O.compose_adjoint(gs[b].astype(np.float64), xs[b].astype(np.float64), passes, border)
        ref_gx.append(a)
        ref_t.append(np.concatenate(t))
    tref = np.sum(ref_t, axis=0)
    assert np.abs(host(tg) - tref).max() <= 2e-5 * np.abs(tref).max()
    gref = np.stack(ref_gx).reshape(shape)
    assert np.abs(host(gx.tensor()) - gref).max() <= 2e-6 * np.abs(gref).max()


@pytest.mark.parametrize("tdt", [torch.bfloat16, torch.float16])
@pytest.mark.parametrize("k", [3, 5, 7, 9])
@pytest.mark.parametrize("border", [0, 2])
def test_small_filter_gradients_16bit(tdt, k, border):
    """16-bit storage of X, G and dL/dX for small volume filters: dL/dX within
    4e-3 of the stencil magnitude, the tap gradients within 1e-4 of the
    largest, both against the FP64 oracle on the decoded values."""
    rng = np.random.default_rng(500 + k + border)
    shape = (2, 21, 30, 70)
    x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(tdt)
    g = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).to(tdt)
    passes = [(a, rng.standard_normal(k)) for a in range(3)]
    xi, gi = Image.from_tensor(x.cuda()), Image.from_tensor(g.cuda())
    gx = Image.empty(gi.extent(), tdt)
    tg = torch.zeros(3 * k, dtype=torch.float64, device=DEV)
    n.convolve_axes_adjoint(gi, xi, gx, passes, border, tg)
    xd, gd = x.float().numpy().astype(np.float64), g.float().numpy().astype(np.float64)
    ref_gx, ref_t, mag = [], [], []
    for b in range(2):
        a, t = O.compose_adjoint(gd[b], xd[b], passes, border)
        ref_gx.append(a)
        ref_t.append(np.concatenate(t))
        m = np.abs(gd[b])
        for ax, w in passes[::-1]:
            m = O.axis_pass_adjoint(m, ax, np.abs(w), border)
        mag.append(m)
    got = gx.tensor().float().cpu().numpy().astype(np.float64)
    assert (np.abs(got - np.stack(ref_gx)) <= 4e-3 * np.stack(mag) + 1e-30).all()
    tref = np.sum(ref_t, axis=0)
    assert np.abs(host(tg) - tref).max() <= 1e-4 * np.abs(tref).max()


@pytest.mark.parametrize("kshape", [(3, 3), (4, 5), (7, 7), (2, 9), (3, 3, 3), (5, 4, 3), (1, 3, 5), (9, 2, 2)])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_full_kernel_f32_stencil(kshape, border):
    """convolve() with a dense (non-separable) kernel of up to 9 taps per
    axis on f32 images and volumes: the tiled stencil, through a mirrored,
    axis-swapped view, within 1e-6 of the stencil magnitude of the FP64
    oracle (kernel shapes in numpy order: the last is ndl axis 0)."""
    rng = np.random.default_rng(sum(kshape) * 7 + border)
    shape = (77, 130) if len(kshape) == 2 else (19, 30, 45)
    x = rng.standard_normal(shape).astype(np.float32)
    k = rng.standard_normal(kshape)
    k[np.abs(k) < 1e-3] = 0.5                       # dense: no zero tap
    base = Image.from_tensor(dev(x))
    src = base.swap_axes(0, 1).mirror(0)
    logical = src.tensor().cpu().numpy()
    o = Image.empty(src.extent(), torch.float32)
    n.convolve(src, o, k, border)
    ref = O.convolve_total(logical, k, border)
    mag = O.convolve_total(np.abs(logical.astype(np.float64)), np.abs(k), border)
    assert_close(host(o.tensor()), ref, mag, 1e-6, "stencil %s border %d" % (kshape, border))


@pytest.mark.parametrize("dt,odt", [(np.uint8, np.uint8), (np.int16, np.int32), (np.int16, np.float32),
                                    (np.uint8, np.float64)])
@pytest.mark.parametrize("kshape", [(3, 3), (5, 4), (9, 9), (3, 3, 3), (1, 5, 5), (4, 2, 3)])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_full_kernel_integral_exact(dt, odt, kshape, border):
    """convolve() with a full 2-D / 3-D kernel on integral sources of up to
    16 bits: the exact tiled stencil, bit for bit with the oracle's double
    sequence and DstT cast (truncation), zero taps and a mirrored view
    included."""
    rng = np.random.default_rng(sum(kshape) + 3 * border + np.dtype(dt).itemsize)
    shape = (70, 90) if len(kshape) == 2 else (17, 26, 33)
    lo, hi = (0, 250) if dt == np.uint8 else (-300, 300)
    x = rng.integers(lo, hi, shape).astype(dt)
    k = rng.standard_normal(kshape)
    k[rng.random(kshape) < 0.15] = 0.0
    v = Image.from_tensor(dev(x)).mirror(0)
    logical = v.tensor().cpu().numpy()
    o = Image.empty(v.extent(), torch.from_numpy(np.zeros(1, odt)).dtype)
    # a float32 result accumulates in FP32 by default; EXACT asks for the
    # reference's double sequence there too
    n.convolve(v, o, k, border, precision=abi.PREC_EXACT if odt == np.float32 else abi.PREC_AUTO)
    ref = O.cast(O.convolve_total(logical, k, border), O.dtype_code(np.zeros(1, odt)), O.STORE_CAST)
    assert (host(o.tensor()) == ref).all()


@pytest.mark.parametrize("dt,odt", [(np.uint8, np.uint8), (np.int16, np.int32), (np.uint8, np.float64)])
@pytest.mark.parametrize("sigma", [0.8, 1.5, 3.0, 6.0])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_gaussian_blur_integral_image_exact(dt, odt, sigma, border):
    """gaussian_blur of 2-D integral images: the fused exact kernel (x pass
    and y pass in the reference's double arithmetic, one final round), bit
    for bit with the oracle, through a mirrored, transposed view."""
    rng = np.random.default_rng(int(sigma * 10) + 3 * border)
    lo, hi = (0, 256) if dt == np.uint8 else (-400, 400)
    x = rng.integers(lo, hi, (83, 150)).astype(dt)
    v = Image.from_tensor(dev(x)).swap_axes(0, 1).mirror(1)
    logical = v.tensor().cpu().numpy()
    o = Image.empty(v.extent(), torch.from_numpy(np.zeros(1, odt)).dtype)
    n.gaussian_blur(v, o, sigma, border)
    ref = O.gaussian_blur(logical, sigma, border, O.dtype_code(np.zeros(1, odt)))
    assert (host(o.tensor()) == ref).all()


@pytest.mark.parametrize("border", [0, 1, 2])
def test_gaussian_blur_axes_integral_image_exact(border):
    """gaussian_blur_axes with a different sigma per axis on a 2-D uint8
    image: the fused exact kernel, bit for bit with the oracle's gaussian
    structure (one final round)."""
    rng = np.random.default_rng(40 + border)
    x = rng.integers(0, 256, (97, 131)).astype(np.uint8)
    s = Image.from_tensor(dev(x))
    o = Image.empty(s.extent(), torch.uint8)
    n.gaussian_blur_axes(s, o, [1.3, 2.7], border)
    ref = O.compose(x, [(0, O.gaussian_weights(1.3)), (1, O.gaussian_weights(2.7))], border, O.U8, O.STORE_ROUND)
    assert (host(o.tensor()) == ref).all()


@pytest.mark.parametrize("dt,odt", [(np.uint8, np.uint8), (np.int16, np.int16), (np.uint8, np.float64)])
@pytest.mark.parametrize("sigma", [0.8, 2.0, 3.5])
@pytest.mark.parametrize("border", [0, 1, 2])
def test_gaussian_blur_integral_volume_exact(dt, odt, sigma, border):
    """gaussian_blur of 3-D integral volumes: x and y passes fused in the
    reference's double arithmetic, then the z pass and one final round;
    bit for bit with the oracle, through a mirrored view."""
    rng = np.random.default_rng(int(sigma * 10) + 5 * border)
    lo, hi = (0, 256) if dt == np.uint8 else (-400, 400)
    x = rng.integers(lo, hi, (23, 41, 57)).astype(dt)
    v = Image.from_tensor(dev(x)).mirror(2).mirror(0)
    logical = v.tensor().cpu().numpy()
    o = Image.empty(v.extent(), torch.from_numpy(np.zeros(1, odt)).dtype)
    n.gaussian_blur(v, o, sigma, border)
    ref = O.gaussian_blur(logical, sigma, border, O.dtype_code(np.zeros(1, odt)))
    assert (host(o.tensor()) == ref).all()


@pytest.mark.parametrize("border", [0, 1, 2])
def test_gaussian_blur_integral_volume_exact_strided_dst(border):
    """The exact z pass stores through a mirrored, padded destination view;
    z extents that are not a multiple of the kernel's z chunk."""
    rng = np.random.default_rng(31 + border)
    x = rng.integers(0, 256, (13, 30, 37)).astype(np.uint8)
    v = Image.from_tensor(dev(x))
    buf = torch.zeros((13, 30, 40), dtype=torch.uint8, device="cuda")
    ext = v.extent()
    o = Image.from_tensor(buf).view((0, 0, 0), (ext[0] - 1, ext[1] - 1, ext[2] - 1)).mirror(2).mirror(0)
    assert o.extent() == ext
    n.gaussian_blur(v, o, 1.7, border)
    ref = O.gaussian_blur(x, 1.7, border, O.U8)
    assert (host(o.tensor()) == ref).all()
