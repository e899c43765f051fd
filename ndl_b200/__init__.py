"""ndl_b200 -- B200-native separable N-D convolution, a drop-in for the
convolve() / gaussian_blur() hot path of the ndl image library.

The compute path is libndlgpu.so (hand-written sm_100a CUDA behind the C ABI
of include/ndlgpu.h); this package is its Python host mirror.
"""
from . import abi
from .abi import NdlGpuError
from .convolution import (convolve, gradient, dog_scale_space, downsample, box_blur, box_blur_workspace_size,
                          convolve_axes, convolve_axes_adjoint,
                          convolve_axes_workspace_size, gaussian_blur, gaussian_blur_axes, gaussian_radius,
                          gaussian_taps)
from .image import BorderMode, Image

__all__ = [
    "abi", "NdlGpuError", "Image", "BorderMode", "convolve", "gaussian_blur", "gaussian_blur_axes",
    "convolve_axes", "convolve_axes_adjoint", "convolve_axes_workspace_size", "gaussian_radius", "gaussian_taps",
    "gradient", "dog_scale_space", "downsample", "box_blur", "box_blur_workspace_size",
]
