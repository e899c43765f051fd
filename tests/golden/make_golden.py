"""Generates tests/golden/*.npz from the UNMODIFIED ndl reference.

Run in a tree where oracle/_ref/libndlref.so has been built from the
reference sources (oracle/build_oracle.py).  Every output here comes from the
reference's own ndl::convolve() / ndl::gaussian_blur()
(processing/convolution.h:52-71, :107-186), called through ref_shim.cpp; the
inputs are seeded and small.  The fixtures let the GPU tests check parity on a
machine without the reference tree.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle import oracle as O  # noqa: E402


def binomial():
    return np.array([1, 4, 6, 4, 1], np.float64) / 16.0


def l1_taps(rng, k):
    w = rng.standard_normal(k)
    return w / np.abs(w).sum()


def save(name, meta, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, meta=np.array(json.dumps(meta)), **arrays)
    print("wrote", path, {k: v.shape for k, v in arrays.items()})


def main():
    if not O.have_reference():
        raise SystemExit("build oracle/_ref/libndlref.so first (python oracle/build_oracle.py)")
    rng = np.random.default_rng(20261203)

    # 1. gaussian_blur, 2-D f32, sigma 2 and 1.3, all borders
    x = rng.random((48, 64), dtype=np.float32)
    outs = {}
    for b in (O.CLAMP, O.WRAP, O.REFLECT):
        for sig in (2.0, 1.3):
            outs["out_b%d_s%s" % (b, str(sig).replace(".", "p"))] = O.ref_gaussian_blur(x, sig, b)
    save("gauss2d_f32", {"kind": "gaussian_blur", "sigmas": [2.0, 1.3], "borders": [0, 1, 2]}, src=x, **outs)

    # 2. u8 256^3-like volume through swap_axes(0,2).mirror(1), binomial, Wrap
    base = rng.integers(0, 256, (20, 24, 28), dtype=np.uint8)   # ndl extent {28,24,20}
    # ndl view: swap_axes(0,2) then mirror(1) -> numpy: transpose then flip
    view = np.ascontiguousarray(base).transpose(2, 1, 0)[:, ::-1, :]
    w = binomial()
    passes = [(0, w), (1, w), (2, w)]
    round_once = O.ref_compose(view, passes, O.WRAP, np.uint8, O.STORE_ROUND)
    cast_each = O.ref_compose(view, passes, O.WRAP, np.uint8, O.STORE_CAST)
    save("u8_binomial_view", {"kind": "compose", "view": "swap_axes(0,2).mirror(1)", "border": O.WRAP},
         base=base, taps=w, round_once=round_once, cast_each=cast_each)

    # 3. f32 random 9-tap per axis, Reflect (round-once structure)
    x3 = rng.standard_normal((14, 16, 18)).astype(np.float32)
    taps3 = np.stack([l1_taps(rng, 9) for _ in range(3)])
    y3 = O.ref_compose(x3, [(0, taps3[0]), (1, taps3[1]), (2, taps3[2])], O.REFLECT, np.float32, O.STORE_ROUND)
    y3d = O.ref_compose(x3, [(0, taps3[0]), (1, taps3[1]), (2, taps3[2])], O.REFLECT, np.float64, O.STORE_ROUND)
    save("f32_rand9_reflect", {"kind": "compose", "border": O.REFLECT}, src=x3, taps=taps3, out=y3, out_f64=y3d)

    # 4. u8 gaussian_blur with non-dyadic weights (the exact double path)
    x4 = rng.integers(0, 256, (33, 40), dtype=np.uint8)
    outs = {}
    for b in (O.CLAMP, O.WRAP, O.REFLECT):
        outs["out_b%d" % b] = O.ref_gaussian_blur(x4, 1.5, b)
    save("u8_gauss_s1p5", {"kind": "gaussian_blur", "sigma": 1.5}, src=x4, **outs)

    # 5. reference unit-test images (image_convolution_tests.cpp:18-66,
    #    composite_tests.cpp:110-131, fft_tests.cpp:168-180)
    img = np.arange(1, 17, dtype=np.int32).reshape(4, 4)
    k3 = np.ones((3, 3), np.int32)
    k5 = np.ones((5, 5), np.int32)
    outs = {}
    for b in (O.CLAMP, O.WRAP, O.REFLECT):
        outs["sum3_b%d" % b] = O.ref_convolve(img, k3, b)
        outs["sum5_b%d" % b] = O.ref_convolve(img, k5, b)
    img54 = np.arange(1, 21, dtype=np.int32).reshape(4, 5)
    kb = np.array([[1, 2, 1], [2, 4, 2], [1, 2, 1]], np.int32)
    outs["composite_wrap"] = O.ref_convolve(img54, kb, O.WRAP)
    fimg = np.array([((i + 1) * 37) % 251 for i in range(16 * 8)], np.float64).reshape(8, 16)
    fk = np.array([[1, 2, 1], [0, 1, 0], [-1, 0, 2]], np.float64)
    outs["fft_wrap"] = O.ref_convolve(fimg, fk, O.WRAP)
    save("unit_known_answers", {"kind": "convolve"}, img=img, img54=img54, kb=kb, fimg=fimg, fk=fk, **outs)

    # 6. 1-D: type_coverage_tests.cpp:141-149 and a gaussian_blur DIM==1 (truncating)
    a = np.array([3, 5, 7, 9], np.float32)
    box = np.full(3, 1.0 / 3.0)
    out_box = O.ref_convolve(a, box, O.CLAMP, np.float32)
    x6 = rng.integers(0, 256, (301,), dtype=np.uint8)
    out_g1 = O.ref_gaussian_blur(x6, 2.0, O.REFLECT)
    save("one_d", {"kind": "1d"}, a=a, box=box, out_box=out_box, x6=x6, out_g1=out_g1)

    # 7. 4-D video-like (t, c, y, x) numpy = ndl extent {x, y, c, t}; axes
    #    x, y, t blurred (sigma 2.5, 2.5, 1.5), channel untouched, Reflect
    x7 = rng.random((6, 3, 20, 24), dtype=np.float32)
    gx, gt = O.gaussian_weights(2.5), O.gaussian_weights(1.5)
    y7 = O.ref_compose(x7, [(0, gx), (1, gx), (3, gt)], O.REFLECT, np.float32, O.STORE_ROUND)
    y7d = O.ref_compose(x7, [(0, gx), (1, gx), (3, gt)], O.REFLECT, np.float64, O.STORE_ROUND)
    save("video4d_f32", {"kind": "compose", "border": O.REFLECT, "sigmas": [2.5, 2.5, 0, 1.5]},
         src=x7, out=y7, out_f64=y7d)

    # 8. u8 single truncating convolve() pass with non-dyadic taps, each axis
    x8 = rng.integers(0, 256, (17, 19, 23), dtype=np.uint8)
    w8 = np.array([0.1, 0.2, 0.4, 0.2, 0.1])
    outs = {}
    for ax in range(3):
        kshape = [1, 1, 1]
        kshape[2 - ax] = 5
        outs["ax%d" % ax] = O.ref_convolve(x8, w8.reshape(kshape), O.REFLECT)
    save("u8_trunc_axis", {"kind": "convolve", "border": O.REFLECT}, src=x8, taps=w8, **outs)


if __name__ == "__main__":
    main()
