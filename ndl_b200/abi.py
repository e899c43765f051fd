"""ctypes binding of libndlgpu.so (the C ABI declared in include/ndlgpu.h).

The shared library is the product path.  There is no fallback: if the library
is missing this module raises on first use, telling the caller to build it
(``python -m ndl_b200.build`` or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libndlgpu.so")

MAX_RANK = 8

# ndlgpu_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_UNSUPPORTED_DTYPE = 2
ERR_EXTENT_MISMATCH = 3
ERR_RADIUS_EXCEEDS_EXTENT = 4
ERR_ALIASING = 5
ERR_INDEX_OVERFLOW = 6
ERR_BAD_SIGMA = 7
ERR_WORKSPACE = 8
ERR_CUDA = 9
ERR_OUT_OF_MEMORY = 10
ERR_TOO_MANY_TAPS = 11
ERR_DEVICE_CHECK = 12

# ndlgpu_dtype
U8, I8, U16, I16, I32, U32, I64, U64, F32, F64, F16, BF16 = range(12)
DTYPE_SIZE = {U8: 1, I8: 1, U16: 2, I16: 2, I32: 4, U32: 4, I64: 8, U64: 8, F32: 4, F64: 8, F16: 2, BF16: 2}

# ndlgpu_border (ndl::BorderMode order)
CLAMP, WRAP, REFLECT = 0, 1, 2
# ndlgpu_compose
ROUND_ONCE, CAST_EACH = 0, 1
# ndlgpu_precision
PREC_AUTO, PREC_FP32, PREC_EXACT = 0, 1, 2


class View(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("rank", ctypes.c_int32),
        ("extent", ctypes.c_int64 * MAX_RANK),
        ("stride", ctypes.c_int64 * MAX_RANK),
    ]


class AxisKernel(ctypes.Structure):
    _fields_ = [
        ("axis", ctypes.c_int32),
        ("ntaps", ctypes.c_int32),
        ("center", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("taps", ctypes.POINTER(ctypes.c_double)),
    ]


class NdlGpuError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("ndlgpu status %d (%s): %s" % (status, STATUS_NAMES.get(status, "?"), message))
        self.status = status


STATUS_NAMES = {
    OK: "ok", ERR_INVALID_ARGUMENT: "invalid argument", ERR_UNSUPPORTED_DTYPE: "unsupported dtype",
    ERR_EXTENT_MISMATCH: "extent mismatch", ERR_RADIUS_EXCEEDS_EXTENT: "radius exceeds extent",
    ERR_ALIASING: "aliasing", ERR_INDEX_OVERFLOW: "index overflow", ERR_BAD_SIGMA: "bad sigma",
    ERR_WORKSPACE: "workspace", ERR_CUDA: "cuda", ERR_OUT_OF_MEMORY: "out of memory",
    ERR_TOO_MANY_TAPS: "too many taps", ERR_DEVICE_CHECK: "device check",
}

# Every symbol include/ndlgpu.h declares, with its ctypes signature.
_VP = ctypes.c_void_p
_PV = ctypes.POINTER(View)
_PK = ctypes.POINTER(AxisKernel)
_I = ctypes.c_int
_SZ = ctypes.c_size_t
SIGNATURES = {
    "ndlgpu_version": (ctypes.c_char_p, []),
    "ndlgpu_status_string": (ctypes.c_char_p, [_I]),
    "ndlgpu_last_error": (ctypes.c_char_p, []),
    "ndlgpu_convolve": (_I, [_PV, _PV, _PV, _I, _VP]),
    "ndlgpu_convolve_ex": (_I, [_PV, _PV, _PV, _I, _I, _VP]),
    "ndlgpu_gradient": (_I, [_PV, _PV, _I, _VP]),
    "ndlgpu_dog_scale_space": (_I, [_PV, _I, ctypes.c_double, _PV, _PV, _VP]),
    "ndlgpu_downsample": (_I, [_PV, _PV, _I, _I, _I, _VP]),
    "ndlgpu_box_blur": (_I, [_PV, _PV, _I, _I, _VP, ctypes.c_size_t, _VP]),
    "ndlgpu_box_blur_workspace_size": (_I, [_PV, _PV, _I, _I, ctypes.POINTER(ctypes.c_size_t)]),
    "ndlgpu_gaussian_blur": (_I, [_PV, _PV, ctypes.c_double, _I, _VP, _SZ, _VP]),
    "ndlgpu_gaussian_blur_workspace_size": (_I, [_PV, _PV, ctypes.c_double, _I, ctypes.POINTER(_SZ)]),
    "ndlgpu_gaussian_blur_axes": (_I, [_PV, _PV, ctypes.POINTER(ctypes.c_double), _I, _VP, _SZ, _VP]),
    "ndlgpu_convolve_axes": (_I, [_PV, _PV, _I, _PK, _I, _I, _I, _VP, _SZ, _VP]),
    "ndlgpu_convolve_axes_workspace_size": (_I, [_PV, _PV, _I, _PK, _I, _I, _I, ctypes.POINTER(_SZ)]),
    "ndlgpu_convolve_axes_adjoint": (_I, [_PV, _PV, _PV, _I, _PK, _I, _VP, _I, _VP, _SZ, _VP]),
    "ndlgpu_convolve_axes_adjoint_workspace_size": (_I, [_PV, _PV, _PV, _I, _PK, _I, _I, ctypes.POINTER(_SZ)]),
    "ndlgpu_device_status": (_I, [_VP, ctypes.POINTER(ctypes.c_int32)]),
    "ndlgpu_test_wait_timeouts": (_I, [_I, _I]),
    "ndlgpu_kernel_launches": (ctypes.c_uint64, []),
    "ndlgpu_gaussian_blur_noalloc": (_I, [_PV, _PV, ctypes.c_double, _I, _VP]),
    "ndlgpu_batch_create": (_I, [ctypes.POINTER(_VP)]),
    "ndlgpu_batch_add": (_I, [_VP, _PV, _PV, _I, _PK, _I, _I]),
    "ndlgpu_batch_plan": (_I, [_VP, _I]),
    "ndlgpu_batch_launch": (_I, [_VP, _VP]),
    "ndlgpu_batch_graph_launch": (_I, [_VP, _VP]),
    "ndlgpu_batch_destroy": (_I, [_VP]),
    "ndlgpu_batch_tile_configs": (_I, []),
    "ndlgpu_batch_tile_config_info": (_I, [_I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "ndlgpu_batch_info": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_int64)]),
}

_lib = None
_lock = threading.Lock()


def load():
    """Loads libndlgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError("libndlgpu.so not found at %s: build it with __graft_entry__.build() "
                                  "or python ndl_b200/build.py" % LIB_PATH)
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(status):
    if status != OK:
        msg = load().ndlgpu_last_error()
        raise NdlGpuError(status, msg.decode() if msg else "")


def make_view(data_ptr, dtype, extent, stride):
    v = View()
    v.data = data_ptr
    v.dtype = dtype
    v.rank = len(extent)
    if not 1 <= v.rank <= MAX_RANK:
        raise ValueError("rank must be 1..8")
    for i, (e, s) in enumerate(zip(extent, stride)):
        v.extent[i] = int(e)
        v.stride[i] = int(s)
    return v


def make_passes(passes):
    """passes: iterable of (axis, taps[, center]); returns (array, keepalive)."""
    passes = list(passes)
    arr = (AxisKernel * len(passes))()
    keep = []
    for i, p in enumerate(passes):
        axis, taps = p[0], [float(t) for t in p[1]]
        center = p[2] if len(p) > 2 and p[2] is not None else len(taps) // 2
        buf = (ctypes.c_double * len(taps))(*taps)
        keep.append(buf)
        arr[i].axis = int(axis)
        arr[i].ntaps = len(taps)
        arr[i].center = int(center)
        arr[i].reserved = 0
        arr[i].taps = ctypes.cast(buf, ctypes.POINTER(ctypes.c_double))
    return arr, keep
