"""torch.autograd binding of the separable convolution chain, through the
same C ABI (ndlgpu_convolve_axes / ndlgpu_convolve_axes_adjoint).

    y = separable_conv(x, taps, axes, border)

applies one 1-D correlation per entry of ``axes`` (ndl axis numbers: axis 0
is the tensor's last dim) with the matching 1-D tap tensor, in order, with
gaussian_blur()'s composition (processing/convolution.h:148-185; for float
data that is plain FP32 or FP64 accumulation).  Gradients flow to ``x`` and
to every tap tensor: the backward pass is the hand-written adjoint kernel
(the border-aware transpose for dL/dx, deterministic block-reduced
correlations for dL/dtaps).  float64 tensors run the FP64 kernels, which is
what torch.autograd.gradcheck needs; float32 tensors run the FP32 kernels.
"""
from __future__ import annotations

import torch

from . import abi
from .convolution import convolve_axes, convolve_axes_adjoint
from .image import Image


def _passes(axes, taps):
    return [(int(a), t.detach().to("cpu", torch.float64).numpy()) for a, t in zip(axes, taps)]


class SeparableConv(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, axes, border, *taps):
        if not x.is_cuda:
            raise ValueError("separable_conv runs on CUDA tensors")
        xc = x.contiguous()
        passes = _passes(axes, taps)
        y = torch.empty_like(xc)
        convolve_axes(Image.from_tensor(xc), Image.from_tensor(y), passes, border)
        ctx.axes, ctx.border = axes, border
        ctx.save_for_backward(xc, *taps)
        return y

    @staticmethod
    def backward(ctx, gy):
        xc, *taps = ctx.saved_tensors
        passes = _passes(ctx.axes, taps)
        need_x = ctx.needs_input_grad[0]
        need_t = any(ctx.needs_input_grad[3:])
        g = gy.contiguous().to(xc.dtype)
        gx = torch.empty_like(xc) if need_x else None
        gt = None
        if need_t:
            gt = torch.zeros(sum(len(w) for _, w in passes), dtype=torch.float64 if xc.dtype == torch.float64
                             else torch.float32, device=xc.device)
        if need_x or need_t:
            convolve_axes_adjoint(Image.from_tensor(g), Image.from_tensor(xc) if need_t else None,
                                  Image.from_tensor(gx) if need_x else None, passes, ctx.border, gt)
        tap_grads = []
        off = 0
        for t in taps:
            k = t.numel()
            tap_grads.append(gt[off:off + k].to(t.dtype).to(t.device).reshape(t.shape) if need_t else None)
            off += k
        return (gx, None, None, *tap_grads)


def separable_conv(x, taps, axes=None, border=abi.CLAMP):
    """x: CUDA tensor (float32/float64); taps: list of 1-D tensors; axes:
    ndl axis per tap tensor (default 0..len(taps)-1)."""
    if axes is None:
        axes = list(range(len(taps)))
    return SeparableConv.apply(x, tuple(int(a) for a in axes), int(border), *taps)
