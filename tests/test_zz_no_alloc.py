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


@pytest.mark.parametrize("dtype,shape,sigma,border,uses_scratch", [
    (torch.uint8, (37, 50, 61), 1.5, BorderMode.Reflect, True),     # exact x/y kernel + z pass: one double volume
    (torch.uint8, (40, 33, 29), 0.02, BorderMode.Wrap, True),       # taps [0,1,0] (exp underflow): one double volume
    (torch.uint8, (4096, 4096), 2.0, BorderMode.Clamp, False),      # exact 2-D kernel: no scratch at 16 M pixels
    (torch.float32, (200, 300), 4.5, BorderMode.Wrap, True),        # FP32 chain of two 29-tap passes (no fused width)
    (torch.float64, (90, 110), 2.0, BorderMode.Clamp, True),        # double chain, one intermediate
])
def test_noalloc_matches_allocating_entry_point(dtype, shape, sigma, border, uses_scratch):
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
        assert (need > 0) == uses_scratch and need <= 16 * 1024 * 1024
        n.gaussian_blur(src, ref, sigma, border)
        _noalloc(src, out, sigma, border)
        torch.cuda.synchronize()
        a, b = ref.tensor().cpu().numpy(), out.tensor().cpu().numpy()
        # same kernels, same order: identical (0 tolerance for every dtype)
        assert np.array_equal(a, b), (call, np.abs(a.astype(np.float64) - b.astype(np.float64)).max())


def test_noalloc_rejects_blurs_beyond_its_scratch():
    # 256^3 uint8 at sigma 1.5 needs one double volume (134 MB) > 16 MiB:
    # refused before any work (the fake addresses below are never dereferenced)
    lib = abi.load()
    sv = abi.make_view(0x10000000, abi.U8, [256, 256, 256], [1, 256, 65536])
    dv = abi.make_view(0x90000000, abi.U8, [256, 256, 256], [1, 256, 65536])
    st = lib.ndlgpu_gaussian_blur_noalloc(ctypes.byref(sv), ctypes.byref(dv), ctypes.c_double(1.5), 0, None)
    assert st == abi.ERR_WORKSPACE
    assert b"16777216" in lib.ndlgpu_last_error()


@pytest.mark.parametrize("dtype,shape,sigma", [
    (torch.uint8, (40, 33, 29), 0.02),
    (torch.uint8, (37, 50, 61), 1.5),
    (torch.uint8, (300, 200), 2.0),
    (torch.int16, (64, 48, 40), 0.8),
    (torch.float32, (200, 300), 4.5),
    (torch.float64, (30, 20, 25), 1.0),
])
def test_workspace_query_matches_the_call(dtype, shape, sigma):
    # a caller-owned workspace of exactly the reported size is enough (a
    # route needing more fails with NDLGPU_ERR_WORKSPACE instead of
    # allocating), and the result equals the library-allocated call's
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    if dtype.is_floating_point:
        x = torch.rand(shape, generator=g, device="cuda", dtype=dtype)
    else:
        x = torch.randint(0, 200, shape, generator=g, device="cuda", dtype=dtype)
    src = Image.from_tensor(x)
    ref = Image.empty(src.extent(), dtype)
    out = Image.empty(src.extent(), dtype)
    need = _needs_scratch(src, out, sigma, BorderMode.Reflect)
    buf = torch.empty(max(need, 256), dtype=torch.uint8, device="cuda")
    n.gaussian_blur(src, ref, sigma, BorderMode.Reflect)
    n.gaussian_blur(src, out, sigma, BorderMode.Reflect, workspace=(buf.data_ptr(), need))
    torch.cuda.synchronize()
    assert torch.equal(ref.tensor(), out.tensor())
