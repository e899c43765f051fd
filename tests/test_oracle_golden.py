"""The oracle pinned to the reference: known answers of the reference's own
unit tests, golden fixtures made by the compiled reference, and (where it is
built) the compiled reference itself on seeded cases."""
import numpy as np
import pytest

from oracle import oracle as O
from conftest import golden


def _i32(total):
    return O.cast(total, O.I32)


def test_known_answers_4x4():
    # unitTests/image_convolution_tests.cpp:18-66
    img = np.arange(1, 17, dtype=np.int32).reshape(4, 4)
    ident = np.array([[0, 0, 0], [0, 1, 0], [0, 0, 0]], np.int32)
    assert (_i32(O.convolve_total(img, ident)) == img).all()
    s3 = np.ones((3, 3), np.int32)
    out = _i32(O.convolve_total(img, s3, O.CLAMP))
    assert out[1, 1] == 1 + 2 + 3 + 5 + 6 + 7 + 9 + 10 + 11
    assert out[0, 0] == 4 * img[0, 0] + 2 * img[0, 1] + 2 * img[1, 0] + img[1, 1]
    wrap = _i32(O.convolve_total(img, s3, O.WRAP))
    assert wrap[0, 0] != out[0, 0]
    s5 = np.ones((5, 5), np.int32)
    assert _i32(O.convolve_total(img, s5, O.REFLECT))[0, 0] != _i32(O.convolve_total(img, s5, O.CLAMP))[0, 0]


def test_known_answers_demo_grid():
    # demo/convolution/convolution.cpp:200-240: 5x5 grid 1..25, 3x3 ones
    grid = np.arange(1, 26, dtype=np.int32).reshape(5, 5)
    s3 = np.ones((3, 3), np.int32)
    assert _i32(O.convolve_total(grid, s3))[2, 2] == 117
    assert _i32(O.convolve_total(grid, s3, O.CLAMP))[0, 0] == 27
    assert _i32(O.convolve_total(grid, s3, O.WRAP))[0, 0] == 99
    assert _i32(O.convolve_total(grid, s3, O.REFLECT))[0, 0] == 27


def test_composite_wrap_sum_identity():
    # unitTests/composite_tests.cpp:105-133
    img = np.arange(1, 21, dtype=np.int32).reshape(4, 5)
    k = np.array([[1, 2, 1], [2, 4, 2], [1, 2, 1]], np.int32)
    out = _i32(O.convolve_total(img, k, O.WRAP))
    assert out.sum() == k.sum() * img.sum()


def test_fft_correlation_convention():
    # unitTests/fft_tests.cpp:164-223: circular cross-correlation (unflipped,
    # centred at K/2) equals convolve(Wrap) to 1e-6
    W, H = 16, 8
    img = np.array([((i + 1) * 37) % 251 for i in range(W * H)], np.float64).reshape(H, W)
    k = np.array([[1, 2, 1], [0, 1, 0], [-1, 0, 2]], np.float64)
    out = O.convolve_total(img, k, O.WRAP)
    pad = np.zeros((H, W))
    for ky in range(3):
        for kx in range(3):
            pad[(ky - 1) % H, (kx - 1) % W] = k[ky, kx]
    corr = np.real(np.fft.ifft2(np.conj(np.fft.fft2(pad)) * np.fft.fft2(img)))
    assert np.abs(corr - out).max() < 1e-6


def test_float_box_1d():
    # unitTests/type_coverage_tests.cpp:141-149
    a = np.array([3, 5, 7, 9], np.float32)
    out = O.cast(O.convolve_total(a, np.full(3, 1.0 / 3.0), O.CLAMP), O.F32)
    assert out[1] == np.float32((3.0 + 5.0 + 7.0) / 3.0)


def test_border_maps():
    # unitTests/image_core_tests.cpp:456-508 (4-wide)
    assert O.border_map(O.CLAMP, 4, -2) == 0
    assert O.border_map(O.WRAP, 4, -2) == 2
    assert O.border_map(O.REFLECT, 4, -2) == 1
    assert O.border_map(O.CLAMP, 4, 5) == 3
    assert O.border_map(O.WRAP, 4, 5) == 1
    assert O.border_map(O.REFLECT, 4, 5) == 2


def test_gaussian_impulse_response():
    # docs/tutorials/convolution_tutorial.md:138-150: gaussian_blur(impulse,
    # response, 1.0) of a 1000 impulse, printed to 2 decimals
    imp = np.zeros((11, 11))
    imp[5, 5] = 1000.0
    r = O.gaussian_blur(imp, 1.0)
    row5 = [0.00, 0.00, 1.77, 21.55, 96.58, 159.24, 96.58, 21.55, 1.77, 0.00, 0.00]
    row3 = [0.00, 0.00, 0.24, 2.92, 13.07, 21.55, 13.07, 2.92, 0.24, 0.00, 0.00]
    assert np.allclose(np.round(r[5], 2), row5)
    assert np.allclose(np.round(r[3], 2), row3)
    assert O.gaussian_radius(1.0) == 3 and O.gaussian_radius(2.0) == 6 and O.gaussian_radius(6.0) == 18


@pytest.mark.parametrize("name", ["gauss2d_f32", "u8_gauss_s1p5"])
def test_oracle_matches_golden_gaussian(name):
    d, meta = golden(name)
    src = d["src"]
    for key in d.files:
        if not key.startswith("out_b"):
            continue
        b = int(key[5])
        sig = meta.get("sigma")
        if sig is None:
            sig = float(key.split("_s")[1].replace("p", "."))
        ours = O.gaussian_blur(src, sig, b)
        assert ours.dtype == d[key].dtype
        assert (ours == d[key]).all(), key


def test_oracle_matches_golden_u8_view():
    d, meta = golden("u8_binomial_view")
    view = d["base"].transpose(2, 1, 0)[:, ::-1, :]
    w = d["taps"]
    passes = [(0, w), (1, w), (2, w)]
    assert (O.compose(view, passes, O.WRAP, O.U8, O.STORE_ROUND) == d["round_once"]).all()
    assert (O.compose(view, passes, O.WRAP, O.U8, O.STORE_CAST) == d["cast_each"]).all()
    # the two modes really differ (truncate per pass vs round once)
    assert (d["round_once"] != d["cast_each"]).mean() > 0.5


def test_oracle_matches_golden_float_chains():
    d, _ = golden("f32_rand9_reflect")
    t = d["taps"]
    passes = [(0, t[0]), (1, t[1]), (2, t[2])]
    assert (O.compose(d["src"], passes, O.REFLECT, O.F32) == d["out"]).all()
    assert (O.compose_total(d["src"], passes, O.REFLECT) == d["out_f64"]).all()
    d, _ = golden("video4d_f32")
    gx, gt = O.gaussian_weights(2.5), O.gaussian_weights(1.5)
    passes = [(0, gx), (1, gx), (3, gt)]
    assert (O.compose_total(d["src"], passes, O.REFLECT) == d["out_f64"]).all()


def test_oracle_matches_golden_unit_and_1d():
    d, _ = golden("unit_known_answers")
    for b in (0, 1, 2):
        assert (_i32(O.convolve_total(d["img"], np.ones((3, 3)), b)) == d["sum3_b%d" % b]).all()
        assert (_i32(O.convolve_total(d["img"], np.ones((5, 5)), b)) == d["sum5_b%d" % b]).all()
    assert (_i32(O.convolve_total(d["img54"], d["kb"], O.WRAP)) == d["composite_wrap"]).all()
    assert (O.convolve_total(d["fimg"], d["fk"], O.WRAP) == d["fft_wrap"]).all()
    d, _ = golden("one_d")
    assert (O.cast(O.convolve_total(d["a"], d["box"]), O.F32) == d["out_box"]).all()
    assert (O.gaussian_blur(d["x6"], 2.0, O.REFLECT) == d["out_g1"]).all()
    d, _ = golden("u8_trunc_axis")
    for ax in range(3):
        assert (O.compose(d["src"], [(ax, d["taps"])], O.REFLECT, O.U8) == d["ax%d" % ax]).all()


def test_adjoint_oracle_is_the_transpose():
    """<P x, g> == <x, P^T g> for each border, and tap gradients equal the
    finite-difference derivative (exact for a linear map)."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal((7, 9, 11))
    g = rng.standard_normal((7, 9, 11))
    w = rng.standard_normal(5)
    for b in (O.CLAMP, O.WRAP, O.REFLECT):
        for ax in range(3):
            lhs = (O.axis_pass_total(x, ax, w, b) * g).sum()
            rhs = (x * O.axis_pass_adjoint(g, ax, w, b)).sum()
            assert abs(lhs - rhs) < 1e-9 * (abs(lhs) + 1)
            tg = O.axis_tap_grad(g, x, ax, len(w), b)
            for k in range(len(w)):
                e = np.zeros_like(w)
                e[k] = 1.0
                assert abs(tg[k] - (O.axis_pass_total(x, ax, e, b) * g).sum()) < 1e-9 * (abs(tg[k]) + 1)


@pytest.mark.skipif(not O.have_reference(), reason="compiled reference not present")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_compiled_reference_random(seed):
    rng = np.random.default_rng(seed)
    shape = tuple(int(v) for v in rng.integers(3, 12, size=int(rng.integers(1, 4))))
    b = int(rng.integers(0, 3))
    for dt in (np.uint8, np.int16, np.float32, np.float64):
        if np.issubdtype(dt, np.integer):
            x = rng.integers(0, 100, shape).astype(dt)
        else:
            x = rng.standard_normal(shape).astype(dt)
        kshape = tuple(int(v) for v in rng.integers(1, min(shape) + 1, size=len(shape)))
        k = rng.standard_normal(kshape)
        k[rng.random(kshape) < 0.2] = 0.0
        ref = O.ref_convolve(x, k, b)
        ours = O.cast(O.convolve_total(x, k, b), O.dtype_code(x))
        assert (ref == ours).all() or (np.isnan(ref) == np.isnan(ours)).all()
        sig = float(rng.uniform(0.4, 1.2))
        if b == O.CLAMP or 2 * O.gaussian_radius(sig) < min(shape):
            assert (O.ref_gaussian_blur(x, sig, b) == O.gaussian_blur(x, sig, b)).all()


@pytest.mark.skipif(not O.have_reference(), reason="compiled reference not present")
@pytest.mark.parametrize("shape", [(17,), (9, 13), (5, 7, 11)])
def test_gradient_oracle_matches_compiled_reference(shape):
    """The oracle's gradient() (convolve with {-0.5, 0, +0.5} per axis, cast
    as convolve casts) against ndl::gradient() itself, bit for bit."""
    rng = np.random.default_rng(len(shape))
    for dt, odt in [(np.float32, np.float32), (np.uint8, np.int16), (np.int32, np.int32), (np.float64, np.float64),
                    (np.uint8, np.float32)]:
        x = rng.standard_normal(shape).astype(dt) if dt in (np.float32, np.float64) else \
            (rng.random(shape) * 200).astype(dt)
        for border in (0, 1, 2):
            r = O.ref_gradient(x, border, odt)
            o = O.gradient(x, border, O.dtype_code(np.zeros(1, odt)))
            assert (r == o).all(), (dt, odt, border)


def blob_image(shape, n, seed):
    """Seeded Gaussian blobs of both signs (sigma 1.5-4, amplitude up to 120)
    over U[0, 4) noise: an image with many DoG extrema."""
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    x = rng.random(shape) * 4.0
    for _ in range(n):
        c = [rng.uniform(0, s) for s in shape]
        sg = rng.uniform(1.5, 4.0)
        x += rng.uniform(-120, 120) * np.exp(-sum((g - ci) ** 2 for g, ci in zip(grids, c)) / (2 * sg * sg))
    return x


@pytest.mark.skipif(not O.have_reference(), reason="compiled reference not present")
@pytest.mark.parametrize("shape,ns,s0", [((64, 72), 5, 1.6), ((48, 56), 6, 1.2), ((24, 26, 28), 4, 0.8)])
def test_dog_oracle_matches_detect_keypoints(shape, ns, s0):
    """The oracle's scale space (sigma schedule, Reflect blurs in double,
    level differences), run through the restated extrema search, gives
    exactly the keypoints of ndl::detect_keypoints() itself: the same
    positions, the same scales and bit-identical |DoG| responses."""
    x = blob_image(shape, 40, sum(shape))
    for thr in (0.5, 5.0):
        ref = O.ref_detect_keypoints(x, ns, s0, thr)
        _, dogs = O.dog_scale_space(x, ns, s0)
        ours = O.dog_keypoints(dogs, O.dog_sigmas(ns, s0), thr)
        assert len(ref) >= 5
        assert ref == ours


def test_downsample_known_answers():
    """image_convolution_tests.cpp:70-92: a constant {3, 40, 30} uint8 colour
    image (channel axis 0) downsamples by 2 to {3, 20, 15}, still constant."""
    x = np.full((30, 40, 3), 77, np.uint8)           # ndl extent {3, 40, 30}
    out = O.downsample(x, 2, 0)
    assert out.shape == (15, 20, 3) and (out == 77).all()
    # a short last block averages only the samples that exist (:273-277)
    y = np.arange(10, dtype=np.float64).reshape(2, 5)  # ndl {5, 2}; channel axis 1
    assert (O.downsample(y, 2, 1) == np.array([[0.5, 2.5, 4.0], [5.5, 7.5, 9.0]])).all()


@pytest.mark.skipif(not O.have_reference(), reason="compiled reference not present")
@pytest.mark.parametrize("shape,factor,ch", [((30, 40, 3), 2, 0), ((31, 17, 3), 3, 0), ((9, 10, 11), 4, 1),
                                             ((5, 7, 9, 2), 2, 3), ((33, 21), 5, 1), ((6, 50), 7, 0)])
def test_downsample_oracle_matches_compiled_reference(shape, factor, ch):
    rng = np.random.default_rng(factor + ch)
    for dt in (np.uint8, np.int16, np.int32, np.float32, np.float64):
        if np.issubdtype(dt, np.integer):
            x = (rng.random(shape) * 250 - (120 if dt != np.uint8 else 0)).astype(dt)
        else:
            x = rng.standard_normal(shape).astype(dt)
        assert (O.ref_downsample(x, factor, ch) == O.downsample(x, factor, ch)).all(), dt


@pytest.mark.skipif(not O.have_reference(), reason="compiled reference not present")
@pytest.mark.parametrize("shape,ch", [((30, 40, 3), 0), ((3, 17, 29), 2), ((40, 3), 0), ((12, 13, 14, 2), 0)])
def test_per_channel_blur_oracle_matches_compiled_reference(shape, ch):
    """per_channel(src, dst, channelAxis, gaussian_blur) (image/kernels.h:78-87)
    is gaussian_blur's structure over the other axes -- with a single other
    axis, the plain truncating convolve() of gaussian_blur's 1-D branch."""
    rng = np.random.default_rng(len(shape) + ch)
    for dt in (np.uint8, np.int16, np.float32):
        x = (rng.random(shape) * 200).astype(dt)
        for b in (0, 1, 2):
            assert (O.ref_per_channel_blur(x, 1.3, ch, b) == O.per_channel_blur(x, 1.3, ch, b)).all(), (dt, b)


@pytest.mark.skipif(not O.have_reference(), reason="compiled reference not present")
@pytest.mark.parametrize("shape", [(17,), (20, 23), (9, 10, 11), (5, 6, 7, 4)])
def test_box_blur_oracle_matches_compiled_reference(shape):
    """box_blur (summed_area_table.h:300-339): padded copy, double table
    built axis by axis, corner inclusion-exclusion, then the cast -- bit for
    bit, floating types included (the running sums keep the reference's
    order)."""
    rng = np.random.default_rng(len(shape))
    for dt, odt in [(np.uint8, np.uint8), (np.float32, np.float32), (np.float64, np.float64), (np.int16, np.float32)]:
        x = (rng.random(shape) * 200).astype(dt) if dt != np.float64 else rng.standard_normal(shape)
        for r in (1, 2, 3):
            for b in (0, 1, 2):
                if r > min(shape) and b != 0:
                    continue
                ref = O.ref_box_blur(x, r, b, odt)
                assert (ref == O.box_blur(x, r, b, O.dtype_code(np.zeros(1, odt)))).all(), (dt, r, b)
