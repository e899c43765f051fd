"""numpy front end of the oracle (TEST INFRASTRUCTURE ONLY).

Two checkers live behind this module:

* the plain-C FP64 restatement in ``ndl_oracle.c`` (always available), and
* the UNMODIFIED reference compiled by ``build_oracle.py`` into
  ``_ref/libndlref.so`` (available where it was built; ``have_reference()``).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this module.  The product library never imports it.

Array convention: a numpy array of shape ``(n_{D-1}, ..., n_1, n_0)`` is the
ndl image of extent ``{n_0, n_1, ..., n_{D-1}}`` -- ndl axis 0 is numpy's last
axis (ndl's default layout has axis 0 fastest, image/core.h:858-864).  Any
numpy view (transposed, reversed, strided) is a valid ndl view of the same
logical content.

bfloat16 has no numpy dtype; such data is carried as ``np.uint16`` bit
patterns together with an explicit ``dtype_code`` of ``BF16``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CLAMP, WRAP, REFLECT = 0, 1, 2
STORE_CAST, STORE_ROUND = 0, 1
U8, I8, U16, I16, I32, U32, I64, U64, F32, F64, F16, BF16 = range(12)

_NP_CODE = {
    np.dtype(np.uint8): U8, np.dtype(np.int8): I8, np.dtype(np.uint16): U16,
    np.dtype(np.int16): I16, np.dtype(np.int32): I32, np.dtype(np.uint32): U32,
    np.dtype(np.int64): I64, np.dtype(np.uint64): U64, np.dtype(np.float32): F32,
    np.dtype(np.float64): F64, np.dtype(np.float16): F16,
}
_CODE_NP = {v: k for k, v in _NP_CODE.items()}
_CODE_NP[BF16] = np.dtype(np.uint16)

_lib = None
_ref = None

_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "libndloracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run oracle/build_oracle.py")
        _lib = ctypes.CDLL(path)
        for name in ("ora_convolve", "ora_axis_pass", "ora_axis_pass_adjoint", "ora_axis_tap_grad", "ora_downsample",
                     "ora_box_blur"):
            getattr(_lib, name).restype = ctypes.c_int
        _lib.ora_gaussian_weights.restype = ctypes.c_int
        _lib.ora_gaussian_weights.argtypes = [ctypes.c_double, _f64p]
        _lib.ora_gaussian_radius.restype = ctypes.c_int
        _lib.ora_gaussian_radius.argtypes = [ctypes.c_double]
        _lib.ora_border_map.restype = ctypes.c_int
        _lib.ora_border_map.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64]
        _lib.ora_cast.restype = ctypes.c_int
    return _lib


def reference_path():
    return os.path.join(HERE, "_ref", "libndlref.so")


def have_reference():
    return os.path.exists(reference_path())


def _load_ref():
    global _ref
    if _ref is None:
        if not have_reference():
            raise RuntimeError("reference shim not built (oracle/build_oracle.py needs the ndl source tree)")
        _ref = ctypes.CDLL(reference_path())
        for name in ("ref_convolve", "ref_gaussian_blur", "ref_compose", "ref_view_probe", "ref_gradient",
                     "ref_detect_keypoints", "ref_downsample", "ref_per_channel_blur", "ref_box_blur"):
            getattr(_ref, name).restype = ctypes.c_int
    return _ref


def dtype_code(a, code=None):
    if code is not None:
        return code
    return _NP_CODE[np.dtype(a.dtype)]


def to_f64(a, code=None):
    """Decode any supported array to float64 (logical content preserved)."""
    code = dtype_code(a, code)
    if code == BF16:
        bits = np.ascontiguousarray(a).astype(np.uint32) << 16
        return bits.view(np.float32).astype(np.float64)
    return np.ascontiguousarray(a).astype(np.float64)


def _ndl_geom(a):
    """(extent, stride) in ndl axis order, strides in elements."""
    item = a.dtype.itemsize
    ext = list(a.shape[::-1])
    st = [s // item for s in a.strides[::-1]]
    return ext, st


def _arr64(vals):
    return (ctypes.c_int64 * len(vals))(*vals)


# ----------------------------------------------------------------------------
# FP64 restatement
# ----------------------------------------------------------------------------

def border_map(border, M, x):
    return _load().ora_border_map(border, M, x)


def gaussian_radius(sigma):
    """_kernelSize(sigma), mathHelpers.h:17-18."""
    return _load().ora_gaussian_radius(float(sigma))


def gaussian_weights(sigma):
    """Normalised taps of processing/convolution.h:116-126."""
    r = gaussian_radius(sigma)
    w = np.zeros(2 * r + 1, np.float64)
    _load().ora_gaussian_weights(float(sigma), w.ctypes.data_as(_f64p))
    return w


def convolve_total(src, kernel, border=CLAMP, code=None):
    """Double totals of convolve(src, ., kernel, border) (before the DstT
    cast).  ``kernel`` is a numpy array in the same reversed axis order."""
    x = to_f64(src, code)
    k = np.ascontiguousarray(kernel, dtype=np.float64)
    if k.ndim != x.ndim:
        raise ValueError("kernel rank must equal image rank")
    out = np.zeros_like(x)
    ext, st = _ndl_geom(x)
    _, ost = _ndl_geom(out)
    kext = list(k.shape[::-1])
    rc = _load().ora_convolve(x.ndim, x.ctypes.data_as(_f64p), _arr64(ext), _arr64(st),
                              out.ctypes.data_as(_f64p), _arr64(ost),
                              k.ctypes.data_as(_f64p), _arr64(kext), border)
    if rc != 0:
        raise RuntimeError("ora_convolve failed")
    return out


def axis_pass_total(x, axis, w, border=CLAMP, center=None):
    """Double totals of one 1-D pass along ndl axis ``axis`` of a float64
    array (tap k reads offset k - center; center defaults to K/2)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    K = len(w)
    c = K // 2 if center is None else center
    out = np.zeros_like(x)
    ext, st = _ndl_geom(x)
    _, ost = _ndl_geom(out)
    rc = _load().ora_axis_pass(x.ndim, x.ctypes.data_as(_f64p), _arr64(ext), _arr64(st),
                               out.ctypes.data_as(_f64p), _arr64(ost),
                               axis, K, c, w.ctypes.data_as(_f64p), border)
    if rc != 0:
        raise RuntimeError("ora_axis_pass failed")
    return out


def axis_pass_adjoint(g, axis, w, border=CLAMP, center=None):
    g = np.ascontiguousarray(g, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    K = len(w)
    c = K // 2 if center is None else center
    out = np.zeros_like(g)
    ext, st = _ndl_geom(g)
    _, ost = _ndl_geom(out)
    rc = _load().ora_axis_pass_adjoint(g.ndim, g.ctypes.data_as(_f64p), _arr64(ext), _arr64(st),
                                       out.ctypes.data_as(_f64p), _arr64(ost),
                                       axis, K, c, w.ctypes.data_as(_f64p), border)
    if rc != 0:
        raise RuntimeError("ora_axis_pass_adjoint failed")
    return out


def axis_tap_grad(g, x, axis, K, border=CLAMP, center=None):
    g = np.ascontiguousarray(g, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    c = K // 2 if center is None else center
    out = np.zeros(K, np.float64)
    ext, st = _ndl_geom(g)
    _, xst = _ndl_geom(x)
    rc = _load().ora_axis_tap_grad(g.ndim, g.ctypes.data_as(_f64p), _arr64(ext), _arr64(st),
                                   x.ctypes.data_as(_f64p), _arr64(xst),
                                   axis, K, c, border, out.ctypes.data_as(_f64p))
    if rc != 0:
        raise RuntimeError("ora_axis_tap_grad failed")
    return out


def cast(total, out_code, mode=STORE_CAST):
    """DstT conversion of double totals: static_cast (convolution.h:69) or
    std::round-then-cast for integral DstT (convolution.h:184)."""
    t = np.ascontiguousarray(total, dtype=np.float64)
    out = np.empty(t.shape, _CODE_NP[out_code])
    rc = _load().ora_cast(t.ctypes.data_as(_f64p), ctypes.c_int64(t.size), out_code, mode,
                          out.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError("ora_cast failed")
    return out


def gradient(src, border=REFLECT, out_code=None, code=None):
    """ndl::gradient (processing/convolution.h:359-388) restated: for every
    ndl axis a, convolve() with the taps {-0.5, 0, +0.5} along a, cast as
    convolve() casts (truncating for integral DstT).  Returns src.shape +
    (DIM,): the leading ndl component axis is the last numpy axis."""
    code = dtype_code(src, code)
    out_code = code if out_code is None else out_code
    x = to_f64(src, code)
    dim = x.ndim
    comps = []
    for a in range(dim):
        kshape = [1] * dim
        kshape[dim - 1 - a] = 3
        k = np.zeros(kshape)
        k.flat[0], k.flat[2] = -0.5, 0.5
        comps.append(cast(convolve_total(x, k, border), out_code, STORE_CAST))
    return np.stack(comps, axis=-1)


def compose(src, passes, border=CLAMP, out_code=F32, mode=STORE_ROUND, code=None):
    """Oracle of a per-axis separable composition.

    passes: list of (ndl_axis, taps) applied in order.
    mode STORE_ROUND: gaussian_blur's structure (processing/convolution.h:
      148-185): double intermediates, one final round (integral) / cast.
      A single pass is a plain convolve() (truncating cast), as in
      gaussian_blur's DIM==1 branch (:141-146).
    mode STORE_CAST: every pass is a full convolve() into DstT (the chain of
      separate convolve() calls).
    """
    x = to_f64(src, code)
    if len(passes) == 1:
        ax, w = passes[0]
        return cast(axis_pass_total(x, ax, w, border), out_code, STORE_CAST)
    if mode == STORE_CAST:
        cur = x
        for ax, w in passes:
            cur = cast(axis_pass_total(cur, ax, w, border), out_code, STORE_CAST)
            cur = to_f64(cur, out_code)
        return cast(cur, out_code, STORE_CAST)
    cur = x
    for ax, w in passes:
        cur = axis_pass_total(cur, ax, w, border)
    return cast(cur, out_code, STORE_ROUND)


def compose_total(src, passes, border=CLAMP, code=None):
    """Double result of the composition before any final cast."""
    cur = to_f64(src, code)
    for ax, w in passes:
        cur = axis_pass_total(cur, ax, w, border)
    return cur


def gaussian_blur(src, sigma, border=CLAMP, out_code=None, code=None):
    """gaussian_blur(src, dst, sigma, border), processing/convolution.h:107-186."""
    w = gaussian_weights(sigma)
    if out_code is None:
        out_code = dtype_code(src, code)
    ndim = np.asarray(src).ndim
    return compose(src, [(a, w) for a in range(ndim)], border, out_code, STORE_ROUND, code)


def downsample_extent(shape, factor, channel_axis=0):
    """numpy shape of downsample()'s result (channel_axis is an ndl axis)."""
    D = len(shape)
    ext = list(shape[::-1])
    out = [e if a == channel_axis else (e - 1) // factor + 1 for a, e in enumerate(ext)]
    return tuple(out[::-1])


def downsample(src, factor, channel_axis=0, code=None, out_code=None):
    """downsample(src, factor, channelAxis), processing/convolution.h:241-305:
    block averages in double, then std::round for integral types (the result
    type is src's unless out_code is given)."""
    x = to_f64(src, code)
    ext, st = _ndl_geom(x)
    shape = downsample_extent(x.shape, factor, channel_axis)
    out = np.zeros(shape, np.float64)
    rc = _load().ora_downsample(x.ndim, x.ctypes.data_as(_f64p), _arr64(ext), _arr64(st), int(factor),
                                int(channel_axis), out.ctypes.data_as(_f64p))
    if rc != 0:
        raise RuntimeError("ora_downsample failed")
    return cast(out, dtype_code(src, code) if out_code is None else out_code, STORE_ROUND)


def box_blur(src, radius, border=CLAMP, out_code=None, code=None):
    """box_blur(src, dst, radius, border), processing/summed_area_table.h:
    300-339: the reference's summed-area-table arithmetic in double, then a
    static_cast to DstT (truncation for integral types)."""
    x = to_f64(src, code)
    ext, st = _ndl_geom(x)
    out = np.zeros(x.shape, np.float64)
    rc = _load().ora_box_blur(x.ndim, x.ctypes.data_as(_f64p), _arr64(ext), _arr64(st), int(radius), int(border),
                              out.ctypes.data_as(_f64p))
    if rc != 0:
        raise RuntimeError("ora_box_blur failed")
    return cast(out, dtype_code(src, code) if out_code is None else out_code, STORE_CAST)


def dog_sigmas(num_scales, sigma0):
    """sigma_i = sigma0 * 2^(i / (num_scales - 3)), feature_detection.h:105-107."""
    return [sigma0 * 2.0 ** (i / (num_scales - 3)) for i in range(num_scales)]


def dog_scale_space(src, num_scales=5, sigma0=1.6, code=None):
    """Levels and Difference-of-Gaussians of detect_keypoints
    (processing/feature_detection.h:101-122), in double: level i is
    gaussian_blur(src as double, sigma_i, Reflect) (no final cast: double
    output), dog[i] = level[i+1] - level[i].  Returns (levels, dogs)."""
    x = to_f64(src, code)
    levels = []
    for s in dog_sigmas(num_scales, sigma0):
        w = gaussian_weights(s)
        levels.append(compose_total(x, [(a, w) for a in range(x.ndim)], REFLECT))
    return levels, [levels[i + 1] - levels[i] for i in range(num_scales - 1)]


def dog_keypoints(dogs, sigmas, threshold):
    """The extrema search of detect_keypoints (feature_detection.h:131-160):
    on every interior layer, positions with |v| >= threshold that are a strict
    max or min against the 3^D - 1 same-layer and 2 * 3^D adjacent-layer
    neighbours, Clamp at the border.  Returns sorted (position (ndl axis
    order), scale, response) tuples."""
    import itertools
    D = dogs[0].ndim
    out = []
    for layer in range(1, len(dogs) - 1):
        v = dogs[layer]
        pads = [np.pad(dogs[layer + d], 1, mode="edge") for d in (-1, 0, 1)]
        ismax = np.abs(v) >= threshold
        ismin = ismax.copy()
        for d in (-1, 0, 1):
            for off in itertools.product((0, 1, 2), repeat=D):
                if d == 0 and all(o == 1 for o in off):
                    continue
                n = pads[d + 1][tuple(slice(o, o + v.shape[i]) for i, o in enumerate(off))]
                ismax &= n < v
                ismin &= n > v
        for idx in np.argwhere(ismax | ismin):
            out.append((tuple(int(i) for i in idx[::-1]), sigmas[layer], float(abs(v[tuple(idx)]))))
    return sorted(out)


def compose_adjoint(g, x, passes, border=CLAMP):
    """FP64 adjoint of the composition Y = P_n(...P_1(X)) for
    L = sum(g * Y): returns (dL/dX, [dL/dw_p for each pass])."""
    inputs = [np.ascontiguousarray(x, dtype=np.float64)]
    for ax, w in passes[:-1]:
        inputs.append(axis_pass_total(inputs[-1], ax, w, border))
    gcur = np.ascontiguousarray(g, dtype=np.float64)
    tap = [None] * len(passes)
    for p in range(len(passes) - 1, -1, -1):
        ax, w = passes[p]
        tap[p] = axis_tap_grad(gcur, inputs[p], ax, len(w), border)
        gcur = axis_pass_adjoint(gcur, ax, w, border)
    return gcur, tap


# ----------------------------------------------------------------------------
# The compiled reference (oracle/_ref)
# ----------------------------------------------------------------------------

def _i32arr(vals):
    return (ctypes.c_int * len(vals))(*[int(v) for v in vals])


def ref_convolve(src, kernel, border=CLAMP, out_dtype=None, out=None):
    """Runs ndl::convolve() itself.  ``out`` may be a preallocated view."""
    lib = _load_ref()
    if out is None:
        out = np.zeros(src.shape, out_dtype or src.dtype)
    k = np.ascontiguousarray(kernel, dtype=np.float64)
    ext, sst = _ndl_geom(src)
    _, dst = _ndl_geom(out)
    rc = lib.ref_convolve(src.ndim, dtype_code(src), ctypes.c_void_p(src.ctypes.data), _i32arr(ext), _i32arr(sst),
                          dtype_code(out), ctypes.c_void_p(out.ctypes.data), _i32arr(dst),
                          k.ctypes.data_as(_f64p), _i32arr(list(k.shape[::-1])), border)
    if rc != 0:
        raise RuntimeError("ref_convolve failed (%d)" % rc)
    return out


def ref_gradient(src, border=REFLECT, out_dtype=None):
    """Runs ndl::gradient() itself; returns src.shape + (DIM,)."""
    lib = _load_ref()
    out = np.zeros(src.shape + (src.ndim,), out_dtype or src.dtype)
    ext, sst = _ndl_geom(src)
    _, dst = _ndl_geom(out)
    rc = lib.ref_gradient(src.ndim, dtype_code(src), ctypes.c_void_p(src.ctypes.data), _i32arr(ext), _i32arr(sst),
                          dtype_code(out), ctypes.c_void_p(out.ctypes.data), _i32arr(dst), border)
    if rc != 0:
        raise RuntimeError("ref_gradient failed (%d)" % rc)
    return out


def ref_detect_keypoints(src, num_scales=5, sigma0=1.6, threshold=5.0, max_n=100000):
    """Runs ndl::detect_keypoints() itself on src as a double image; returns
    sorted (position (ndl axis order), scale, response) tuples."""
    lib = _load_ref()
    x = np.ascontiguousarray(src, dtype=np.float64)
    D = x.ndim
    pos = np.zeros(max_n * D, np.int32)
    sc = np.zeros(max_n, np.float64)
    rs = np.zeros(max_n, np.float64)
    n = lib.ref_detect_keypoints(D, x.ctypes.data_as(_f64p), _i32arr(x.shape[::-1]), int(num_scales),
                                 ctypes.c_double(sigma0), ctypes.c_double(threshold),
                                 pos.ctypes.data_as(_i32p), sc.ctypes.data_as(_f64p), rs.ctypes.data_as(_f64p),
                                 int(max_n))
    if n < 0:
        raise RuntimeError("more than %d keypoints" % max_n)
    return sorted((tuple(int(v) for v in pos[k * D:(k + 1) * D]), float(sc[k]), float(rs[k])) for k in range(n))


def per_channel_blur(src, sigma, channel_axis, border=CLAMP, code=None):
    """per_channel(src, dst, channelAxis, gaussian_blur(., ., sigma, border))
    (image/kernels.h:78-87): gaussian_blur's structure over every axis but
    the channel axis (one remaining axis: a plain truncating convolve(),
    convolution.h:141-146)."""
    w = gaussian_weights(sigma)
    D = np.asarray(src).ndim
    passes = [(a, w) for a in range(D) if a != channel_axis]
    return compose(src, passes, border, dtype_code(src, code), STORE_ROUND, code)


def ref_per_channel_blur(src, sigma, channel_axis, border=CLAMP):
    """Runs ndl::per_channel() with ndl::gaussian_blur() itself."""
    lib = _load_ref()
    x = np.ascontiguousarray(src)
    out = np.zeros_like(x)
    rc = lib.ref_per_channel_blur(x.ndim, dtype_code(x), ctypes.c_void_p(x.ctypes.data), _i32arr(x.shape[::-1]),
                                  int(channel_axis), ctypes.c_double(sigma), int(border),
                                  ctypes.c_void_p(out.ctypes.data))
    if rc != 0:
        raise RuntimeError("ref_per_channel_blur failed (%d)" % rc)
    return out


def ref_box_blur(src, radius, border=CLAMP, out_dtype=None):
    """Runs ndl::box_blur() itself."""
    lib = _load_ref()
    out = np.zeros(src.shape, out_dtype or src.dtype)
    ext, sst = _ndl_geom(src)
    _, dst = _ndl_geom(out)
    rc = lib.ref_box_blur(src.ndim, dtype_code(src), ctypes.c_void_p(src.ctypes.data), _i32arr(ext), _i32arr(sst),
                          dtype_code(out), ctypes.c_void_p(out.ctypes.data), _i32arr(dst), int(radius), int(border))
    if rc != 0:
        raise RuntimeError("ref_box_blur failed (%d)" % rc)
    return out


def ref_downsample(src, factor, channel_axis=0):
    """Runs ndl::downsample() itself on a contiguous copy of src; returns its
    result (src's dtype)."""
    lib = _load_ref()
    x = np.ascontiguousarray(src)
    out = np.zeros(downsample_extent(x.shape, factor, channel_axis), x.dtype)
    rc = lib.ref_downsample(x.ndim, dtype_code(x), ctypes.c_void_p(x.ctypes.data), _i32arr(x.shape[::-1]),
                            int(factor), int(channel_axis), ctypes.c_void_p(out.ctypes.data))
    if rc != 0:
        raise RuntimeError("ref_downsample failed (%d)" % rc)
    return out


def ref_gaussian_blur(src, sigma, border=CLAMP, out_dtype=None, out=None):
    lib = _load_ref()
    if out is None:
        out = np.zeros(src.shape, out_dtype or src.dtype)
    ext, sst = _ndl_geom(src)
    _, dst = _ndl_geom(out)
    rc = lib.ref_gaussian_blur(src.ndim, dtype_code(src), ctypes.c_void_p(src.ctypes.data), _i32arr(ext), _i32arr(sst),
                               dtype_code(out), ctypes.c_void_p(out.ctypes.data), _i32arr(dst),
                               ctypes.c_double(sigma), border)
    if rc != 0:
        raise RuntimeError("ref_gaussian_blur failed (%d)" % rc)
    return out


def ref_compose(src, passes, border=CLAMP, out_dtype=None, mode=STORE_ROUND, out=None):
    """Reference convolve() calls composed per axis (ref_shim.cpp:ref_compose);
    mode STORE_ROUND = gaussian_blur structure, STORE_CAST = convolve chain."""
    lib = _load_ref()
    if out is None:
        out = np.zeros(src.shape, out_dtype or src.dtype)
    ext, sst = _ndl_geom(src)
    _, dst = _ndl_geom(out)
    axes = [int(a) for a, _ in passes]
    ntaps = [len(w) for _, w in passes]
    taps = np.concatenate([np.asarray(w, np.float64) for _, w in passes])
    rc = lib.ref_compose(src.ndim, dtype_code(src), ctypes.c_void_p(src.ctypes.data), _i32arr(ext), _i32arr(sst),
                         dtype_code(out), ctypes.c_void_p(out.ctypes.data), _i32arr(dst),
                         len(passes), _i32arr(axes), _i32arr(ntaps), taps.ctypes.data_as(_f64p),
                         0 if mode == STORE_ROUND else 1, border)
    if rc != 0:
        raise RuntimeError("ref_compose failed (%d)" % rc)
    return out


def ref_view_probe(base_extent, ops):
    """Runs the reference's Image view builders; ops are tuples
    ('swap', a, b) | ('mirror', a) | ('view', axis, start, end, step).
    Returns (element offset, extent, stride) in ndl axis order."""
    lib = _load_ref()
    enc = []
    for op in ops:
        if op[0] == "swap":
            enc += [1, op[1], op[2]]
        elif op[0] == "mirror":
            enc += [2, op[1], 0]
        elif op[0] == "view":
            enc += [3, op[1], 0, 4, op[2], op[3], 5, op[4], 0]
        else:
            raise ValueError(op)
    dim = len(base_extent)
    off = ctypes.c_longlong(0)
    ext = (ctypes.c_int * dim)()
    st = (ctypes.c_int * dim)()
    rc = lib.ref_view_probe(dim, _i32arr(base_extent), _i32arr(enc), len(enc) // 3,
                            ctypes.byref(off), ext, st)
    if rc != 0:
        raise RuntimeError("ref_view_probe failed (%d)" % rc)
    return off.value, list(ext), list(st)
