"""The allocation-free entry point, ndlgpu_gaussian_blur_noalloc.

It exists for callers that cannot allocate device memory (a plugin inside an
application that owns the GPU's memory pool, a real-time loop that must not
reach the allocator, code held to a static memory budget): it runs the same
blur as ndlgpu_gaussian_blur with the scratch taken from a fixed 16 MiB array
inside the library.  Checked here through the C ABI against the allocating
entry point, on two calls in a row (the array keeps the previous call's
contents), on blurs that do use the scratch.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

import ndl_b200 as n
from ndl_b200 import BorderMode, Image, abi

pytestmark = pytest.mark.gpu


def _noalloc(src, dst, sigma, border):
    lib = abi.load()
    sv, dv = src.abi_view(), dst.abi_view()
    st = lib.ndlgpu_gaussian_blur_noalloc(ctypes.byref(sv), ctypes.byref(dv), ctypes.c_double(sigma), int(border),
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    abi.check(st)


def _needs_scratch(src, dst, sigma, border):
    lib = abi.load()
    sv, dv = src.abi_view(), dst.abi_view()
    nb = ctypes.c_size_t(0)
    abi.check(lib.ndlgpu_gaussian_blur_workspace_size(ctypes.byref(sv), ctypes.byref(dv), ctypes.c_double(sigma),
                                                      int(border), ctypes.byref(nb)))
    return nb.value


@pytest.mark.parametrize("dtype,shape,sigma,border", [
    (torch.uint8, (37, 50, 61), 1.5, BorderMode.Reflect),      # exact double chain: two double volumes
    (torch.float32, (200, 300), 4.5, BorderMode.Wrap),         # FP32 chain of two 29-tap passes (no fused width)
    (torch.float64, (90, 110), 2.0, BorderMode.Clamp),         # double chain, one intermediate
])
def test_noalloc_matches_allocating_entry_point(dtype, shape, sigma, border):
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    for call in range(2):
        if dtype == torch.uint8:
            x = torch.randint(0, 256, shape, generator=g, device="cuda", dtype=dtype)
        else:
            x = torch.rand(shape, generator=g, device="cuda", dtype=dtype)
        src = Image.from_tensor(x)
        ref = Image.empty(src.extent(), dtype)
        out = Image.empty(src.extent(), dtype)
        need = _needs_scratch(src, out, sigma, border)
        assert 0 < need <= 16 * 1024 * 1024
        n.gaussian_blur(src, ref, sigma, border)
        _noalloc(src, out, sigma, border)
        torch.cuda.synchronize()
        a, b = ref.tensor().cpu().numpy(), out.tensor().cpu().numpy()
        # same kernels, same order: identical (0 tolerance for every dtype)
        assert np.array_equal(a, b), (call, np.abs(a.astype(np.float64) - b.astype(np.float64)).max())


def test_noalloc_rejects_blurs_beyond_its_scratch():
    # 256^3 uint8 needs two double volumes (268 MB) > 16 MiB: refused before
    # any work (the fake addresses below are never dereferenced)
    lib = abi.load()
    sv = abi.make_view(0x10000000, abi.U8, [256, 256, 256], [1, 256, 65536])
    dv = abi.make_view(0x90000000, abi.U8, [256, 256, 256], [1, 256, 65536])
    st = lib.ndlgpu_gaussian_blur_noalloc(ctypes.byref(sv), ctypes.byref(dv), ctypes.c_double(1.5), 0, None)
    assert st == abi.ERR_WORKSPACE
    assert b"16777216" in lib.ndlgpu_last_error()
