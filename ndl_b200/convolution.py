"""Python mirror of ndl's convolution toolkit (processing/convolution.h),
running on the B200 through the C ABI of libndlgpu.so.

Same names, argument meaning and defaults as the reference:

* ``convolve(src, dst, kernel, border=BorderMode.Clamp)``
  -- processing/convolution.h:52-71
* ``gaussian_blur(src, dst, sigma, border=BorderMode.Clamp)``
  -- processing/convolution.h:107-186

where ``src``/``dst`` are ``ndl_b200.Image`` views of device memory (any
strides, including the negative ones ``mirror()`` makes) and ``kernel`` is a
host array (numpy or nested list) in the same reversed axis order as
``Image.tensor()`` (numpy dim 0 = ndl axis DIM-1).  The reference reports a
wrong extent with assert(); here every precondition raises ``NdlGpuError``
before any work is enqueued.  Calls are asynchronous on the current torch
CUDA stream unless ``stream`` is given.

Extensions beyond the reference (documented in include/ndlgpu.h):
``gaussian_blur_axes`` (one sigma per axis), ``convolve_axes`` (a chain of
1-D passes with explicit composition and precision) and
``convolve_axes_adjoint`` (input and tap gradients).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import abi
from .image import BorderMode, Image


def _stream_ptr(stream):
    if stream is None:
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, torch.cuda.Stream):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def _host_kernel_view(kernel, rank):
    k = np.ascontiguousarray(np.asarray(kernel))
    if k.dtype == np.bool_:
        k = k.astype(np.uint8)
    code = {np.dtype(np.uint8): abi.U8, np.dtype(np.int8): abi.I8, np.dtype(np.uint16): abi.U16,
            np.dtype(np.int16): abi.I16, np.dtype(np.int32): abi.I32, np.dtype(np.uint32): abi.U32,
            np.dtype(np.int64): abi.I64, np.dtype(np.uint64): abi.U64, np.dtype(np.float32): abi.F32,
            np.dtype(np.float64): abi.F64, np.dtype(np.float16): abi.F16}.get(k.dtype)
    if code is None:
        k = k.astype(np.float64)
        code = abi.F64
    if k.ndim != rank:
        raise ValueError("kernel rank %d != image rank %d" % (k.ndim, rank))
    ext = list(k.shape[::-1])
    st = [s // k.itemsize for s in k.strides[::-1]]
    return abi.make_view(k.ctypes.data, code, ext, st), k


def gradient(src: Image, dst: Image = None, border=BorderMode.Reflect, stream=None):
    """ndl::gradient(src, dst, border): dst.slice(0, a) is the central
    difference along axis a, i.e. convolve() with the taps {-0.5, 0, +0.5}
    along a (processing/convolution.h:359-388).  dst has a leading component
    axis of extent src.dim followed by src's extents; with dst None one is
    made in src's type.  The reference's default border is Reflect."""
    if dst is None:
        dst = Image.empty([src.dim] + list(src.extent()), src.dtype)
    lib = abi.load()
    sv, dv = src.abi_view(), dst.abi_view()
    abi.check(lib.ndlgpu_gradient(ctypes.byref(sv), ctypes.byref(dv), int(border), _stream_ptr(stream)))
    return dst


def box_blur(src: Image, dst: Image, radius: int, border=BorderMode.Clamp, workspace=None, stream=None):
    """ndl::box_blur(src, dst, radius, border)
    (processing/summed_area_table.h:300-339): the (2r+1)^DIM box average
    through the reference's own summed-area-table arithmetic (bit-exact)."""
    lib = abi.load()
    sv, dv = src.abi_view(), dst.abi_view()
    ws, wsb = _ws(workspace)
    abi.check(lib.ndlgpu_box_blur(ctypes.byref(sv), ctypes.byref(dv), int(radius), int(border), ws, wsb,
                                  _stream_ptr(stream)))
    return dst


def box_blur_workspace_size(src: Image, dst: Image, radius: int, border=BorderMode.Clamp):
    """Bytes of the summed-area table box_blur needs (8 per padded element)."""
    lib = abi.load()
    sv, dv = src.abi_view(), dst.abi_view()
    b = ctypes.c_size_t(0)
    abi.check(lib.ndlgpu_box_blur_workspace_size(ctypes.byref(sv), ctypes.byref(dv), int(radius), int(border),
                                                 ctypes.byref(b)))
    return b.value


def downsample(src: Image, factor: int, channel_axis=0, border=BorderMode.Clamp, dst: Image = None, stream=None):
    """ndl::downsample(src, factor, channelAxis, border)
    (processing/convolution.h:241-305): every axis but channel_axis shrinks
    by factor, each output the average of its non-overlapping block (rounded
    for integral types).  Returns dst (made in src's type when None)."""
    ext = [e if a == channel_axis else (e - 1) // factor + 1 for a, e in enumerate(src.extent())]
    if dst is None:
        dst = Image.empty(ext, src.dtype)
    lib = abi.load()
    sv, dv = src.abi_view(), dst.abi_view()
    abi.check(lib.ndlgpu_downsample(ctypes.byref(sv), ctypes.byref(dv), int(factor), int(channel_axis), int(border),
                                    _stream_ptr(stream)))
    return dst


def dog_scale_space(src: Image, num_scales=5, sigma0=1.6, dogs=None, levels=None, dtype=None, stream=None):
    """The Difference-of-Gaussians scale space of ndl::detect_keypoints
    (processing/feature_detection.h:101-122): level i is
    gaussian_blur(src, sigma0 * 2^(i / (num_scales - 3)), Reflect) and
    dogs[i] = level[i+1] - level[i].  ``dogs`` (num_scales - 1 images) and
    ``levels`` (num_scales images, or None: not returned) may be given; made
    ones are contiguous images of ``dtype`` (float32 by default).  Returns
    (dogs, levels)."""
    import torch
    dt = dtype or torch.float32
    if dogs is None:
        dogs = [Image.empty(src.extent(), dt) for _ in range(num_scales - 1)]
    if levels is True:
        levels = [Image.empty(src.extent(), dt) for _ in range(num_scales)]
    if len(dogs) != num_scales - 1 or (levels is not None and len(levels) != num_scales):
        raise ValueError("dog_scale_space needs num_scales - 1 dogs and num_scales levels")
    lib = abi.load()
    sv = src.abi_view()
    dv = (abi.View * len(dogs))(*[d.abi_view() for d in dogs])
    lv = (abi.View * len(levels))(*[lv.abi_view() for lv in levels]) if levels is not None else None
    abi.check(lib.ndlgpu_dog_scale_space(ctypes.byref(sv), int(num_scales), ctypes.c_double(sigma0), lv, dv,
                                         _stream_ptr(stream)))
    return dogs, levels


def convolve(src: Image, dst: Image, kernel, border=BorderMode.Clamp, precision=abi.PREC_AUTO, stream=None):
    """ndl::convolve(src, dst, kernel, border): correlation (kernel not
    flipped), centred at K/2 per axis, zero taps skipped, border-mapped per
    axis; integral DstT truncates (processing/convolution.h:52-71)."""
    lib = abi.load()
    kv, keep = _host_kernel_view(kernel, src.dim)
    sv, dv = src.abi_view(), dst.abi_view()
    abi.check(lib.ndlgpu_convolve_ex(ctypes.byref(sv), ctypes.byref(dv), ctypes.byref(kv), int(border),
                                     int(precision), _stream_ptr(stream)))
    del keep
    return dst


def gaussian_blur(src: Image, dst: Image, sigma: float, border=BorderMode.Clamp, workspace=None, stream=None):
    """ndl::gaussian_blur(src, dst, sigma, border) (processing/convolution.h:107-186)."""
    lib = abi.load()
    sv, dv = src.abi_view(), dst.abi_view()
    ws, wsb = _ws(workspace)
    abi.check(lib.ndlgpu_gaussian_blur(ctypes.byref(sv), ctypes.byref(dv), ctypes.c_double(sigma), int(border),
                                       ws, wsb, _stream_ptr(stream)))
    return dst


def gaussian_blur_axes(src: Image, dst: Image, sigmas, border=BorderMode.Clamp, workspace=None, stream=None):
    """gaussian_blur with one sigma per axis (0 leaves an axis untouched)."""
    lib = abi.load()
    sig = (ctypes.c_double * src.dim)(*[float(s) for s in sigmas])
    sv, dv = src.abi_view(), dst.abi_view()
    ws, wsb = _ws(workspace)
    abi.check(lib.ndlgpu_gaussian_blur_axes(ctypes.byref(sv), ctypes.byref(dv), sig, int(border), ws, wsb,
                                            _stream_ptr(stream)))
    return dst


def convolve_axes(src: Image, dst: Image, passes, border=BorderMode.Clamp, compose=abi.ROUND_ONCE,
                  precision=abi.PREC_AUTO, workspace=None, stream=None):
    """A chain of 1-D passes [(axis, taps[, center]), ...] applied in order."""
    lib = abi.load()
    arr, keep = abi.make_passes(passes)
    sv, dv = src.abi_view(), dst.abi_view()
    ws, wsb = _ws(workspace)
    abi.check(lib.ndlgpu_convolve_axes(ctypes.byref(sv), ctypes.byref(dv), len(arr), arr, int(border),
                                       int(compose), int(precision), ws, wsb, _stream_ptr(stream)))
    del keep
    return dst


def convolve_axes_workspace_size(src: Image, dst: Image, passes, border=BorderMode.Clamp, compose=abi.ROUND_ONCE,
                                 precision=abi.PREC_AUTO):
    lib = abi.load()
    arr, keep = abi.make_passes(passes)
    sv, dv = src.abi_view(), dst.abi_view()
    n = ctypes.c_size_t(0)
    abi.check(lib.ndlgpu_convolve_axes_workspace_size(ctypes.byref(sv), ctypes.byref(dv), len(arr), arr, int(border),
                                                      int(compose), int(precision), ctypes.byref(n)))
    del keep
    return n.value


def convolve_axes_adjoint(grad_out: Image, src, grad_src, passes, border=BorderMode.Clamp, grad_taps=None,
                          workspace=None, stream=None):
    """Gradients of L = sum(grad_out * Y), Y = the ROUND_ONCE chain of
    ``passes`` applied to ``src``: writes dL/dsrc into ``grad_src`` (an Image,
    or None) and dL/dtaps into ``grad_taps`` (a 1-D float32/float64 CUDA
    tensor of sum(ntaps) values, or None; needs ``src``)."""
    lib = abi.load()
    arr, keep = abi.make_passes(passes)
    gv = grad_out.abi_view()
    sv = src.abi_view() if src is not None else None
    xv = grad_src.abi_view() if grad_src is not None else None
    tp, tdt = None, abi.F32
    if grad_taps is not None:
        if not (grad_taps.is_cuda and grad_taps.is_contiguous() and grad_taps.dtype in (torch.float32, torch.float64)):
            raise ValueError("grad_taps must be a contiguous float32/float64 CUDA tensor")
        tp = ctypes.c_void_p(grad_taps.data_ptr())
        tdt = abi.F32 if grad_taps.dtype == torch.float32 else abi.F64
    ws, wsb = _ws(workspace)
    abi.check(lib.ndlgpu_convolve_axes_adjoint(ctypes.byref(gv), ctypes.byref(sv) if sv else None,
                                               ctypes.byref(xv) if xv else None, len(arr), arr, int(border),
                                               tp, tdt, ws, wsb, _stream_ptr(stream)))
    del keep
    return grad_src, grad_taps


def _ws(workspace):
    if workspace is None:
        return None, 0
    if isinstance(workspace, torch.Tensor):
        return ctypes.c_void_p(workspace.data_ptr()), workspace.numel() * workspace.element_size()
    ptr, nbytes = workspace
    return ctypes.c_void_p(int(ptr)), int(nbytes)


def gaussian_radius(sigma: float) -> int:
    """_kernelSize(sigma) = _ceil(3.0f * sigma) (mathHelpers.h:17-18)."""
    num = 3.0 * float(sigma)
    t = int(num)
    return t if float(t) == num else t + (1 if num > 0 else 0)


def gaussian_taps(sigma: float) -> np.ndarray:
    """The normalised taps gaussian_blur builds (processing/convolution.h:116-126)."""
    r = gaussian_radius(sigma)
    d = np.arange(-r, r + 1, dtype=np.float64)
    w = np.exp(-(d * d) / (2 * sigma * sigma))
    s = 0.0
    for x in w:          # summed in index order like the reference
        s += float(x)
    return w / s
