"""The C-ABI library on a machine without a GPU: it loads, exports every
symbol include/*.h declares, and rejects bad calls with status codes before
any CUDA call (these calls never reach the device)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import ndl_b200 as n
from ndl_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"NDLGPU_API\s+[\w\s\*]+?\b(ndlgpu_\w+)\s*\(", text))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = abi.load()
    names = declared_symbols()
    assert len(names) >= 13
    for name in names:
        assert hasattr(lib, name), name
    assert set(abi.SIGNATURES) <= names | set()
    assert lib.ndlgpu_version().startswith(b"ndlgpu")


# Fake, never-dereferenced device addresses: validation fails first.
A, B = 0x100000, 0x900000


def V(ptr, dtype, ext, st=None):
    if st is None:
        st, m = [], 1
        for e in ext:
            st.append(m)
            m *= e
    return abi.make_view(ptr, dtype, ext, st)


def call_axes(src, dst, passes, border=0, compose=0, prec=0):
    lib = abi.load()
    arr, keep = abi.make_passes(passes)
    st = lib.ndlgpu_convolve_axes(ctypes.byref(src), ctypes.byref(dst), len(arr), arr, border, compose, prec,
                                  None, 0, None)
    return st, lib.ndlgpu_last_error().decode()


def test_extent_mismatch():
    st, msg = call_axes(V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 9]), [(0, [1, 2, 1])])
    assert st == abi.ERR_EXTENT_MISMATCH and "extent" in msg


def test_aliasing_rejected():
    st, _ = call_axes(V(A, abi.F32, [64, 8]), V(A + 128, abi.F32, [64, 8]), [(0, [1, 2, 1])])
    assert st == abi.ERR_ALIASING


def test_dst_self_overlap_rejected():
    st, _ = call_axes(V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 8], [1, 4]), [(0, [1, 2, 1])])
    assert st == abi.ERR_INVALID_ARGUMENT


def test_radius_exceeds_extent_for_wrap_and_reflect_only():
    taps = [1.0] * 9    # offsets -4..4 on an axis of extent 3
    for border in (abi.WRAP, abi.REFLECT):
        st, _ = call_axes(V(A, abi.F32, [3, 16]), V(B, abi.F32, [3, 16]), [(0, taps)], border)
        assert st == abi.ERR_RADIUS_EXCEEDS_EXTENT


def test_bad_arguments():
    st, _ = call_axes(V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 8]), [(2, [1.0])])
    assert st == abi.ERR_INVALID_ARGUMENT
    st, _ = call_axes(V(A, 42, [8, 8]), V(B, abi.F32, [8, 8]), [(0, [1.0])])
    assert st == abi.ERR_UNSUPPORTED_DTYPE
    st, _ = call_axes(V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 8]), [(0, [1.0] * 300)])
    assert st == abi.ERR_TOO_MANY_TAPS
    st, _ = call_axes(V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 8]), [(0, [1.0])], border=7)
    assert st == abi.ERR_INVALID_ARGUMENT
    st, _ = call_axes(V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 8]), [(0, [1.0])], compose=5)
    assert st == abi.ERR_INVALID_ARGUMENT
    st, _ = call_axes(V(0, abi.F32, [8, 8]), V(B, abi.F32, [8, 8]), [(0, [1.0])])
    assert st == abi.ERR_INVALID_ARGUMENT
    st, _ = call_axes(V(A, abi.F32, [8, -1]), V(B, abi.F32, [8, -1]), [(0, [1.0])])
    assert st == abi.ERR_INVALID_ARGUMENT


def test_empty_image_is_a_no_op():
    # coordinates() is empty: the reference does nothing (convolution.h:64)
    st, _ = call_axes(V(0, abi.F32, [0, 8]), V(0, abi.F32, [0, 8]), [(0, [1, 2, 1])])
    assert st == abi.OK


def test_gaussian_bad_sigma():
    lib = abi.load()
    s, d = V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 8])
    for sigma in (0.0, -1.0, float("nan"), float("inf")):
        st = lib.ndlgpu_gaussian_blur(ctypes.byref(s), ctypes.byref(d), sigma, 0, None, 0, None)
        assert st == abi.ERR_BAD_SIGMA


def test_workspace_size_query_and_too_small_workspace():
    lib = abi.load()
    s, d = V(A, abi.F64, [64, 64, 8]), V(B, abi.F64, [64, 64, 8])
    sz = ctypes.c_size_t(0)
    st = lib.ndlgpu_gaussian_blur_workspace_size(ctypes.byref(s), ctypes.byref(d), 1.0, 0, ctypes.byref(sz))
    assert st == abi.OK and sz.value >= 2 * 64 * 64 * 8 * 8   # two double scratch volumes
    st = lib.ndlgpu_gaussian_blur(ctypes.byref(s), ctypes.byref(d), 1.0, 0, ctypes.c_void_p(0x5000000), 16, None)
    assert st == abi.ERR_WORKSPACE


def test_adjoint_validation():
    lib = abi.load()
    g, x, gx = V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 8]), V(B + 4096, abi.F32, [8, 8])
    arr, keep = abi.make_passes([(0, [1, 2, 1])])
    st = lib.ndlgpu_convolve_axes_adjoint(ctypes.byref(g), None, None, 1, arr, 0, None, abi.F32, None, 0, None)
    assert st == abi.ERR_INVALID_ARGUMENT
    st = lib.ndlgpu_convolve_axes_adjoint(ctypes.byref(g), None, ctypes.byref(gx), 1, arr, 0,
                                          ctypes.c_void_p(0x7000000), abi.F32, None, 0, None)
    assert st == abi.ERR_INVALID_ARGUMENT   # tap gradients need src
    u8 = V(A, abi.U8, [8, 8])
    st = lib.ndlgpu_convolve_axes_adjoint(ctypes.byref(u8), None, ctypes.byref(gx), 1, arr, 0, None, abi.F32,
                                          None, 0, None)
    assert st == abi.ERR_UNSUPPORTED_DTYPE


def test_convolve_kernel_rank_mismatch():
    lib = abi.load()
    s, d = V(A, abi.F32, [8, 8]), V(B, abi.F32, [8, 8])
    k = np.ones(3)
    kv = abi.make_view(k.ctypes.data, abi.F64, [3], [1])
    assert lib.ndlgpu_convolve(ctypes.byref(s), ctypes.byref(d), ctypes.byref(kv), 0, None) == abi.ERR_INVALID_ARGUMENT
