"""The batched form: many images/volumes of uneven extents, tap counts and
border modes run by one persistent launch (optionally replayed from a CUDA
graph).  Wraps the ndlgpu_batch_* entry points of include/ndlgpu.h.

    b = Batch()
    b.add(src, dst, [(0, wx), (1, wy), (2, wz)], BorderMode.Reflect)
    b.add(src2, dst2, [(0, w), (1, w)], BorderMode.Wrap, adjoint=True)
    b.plan()            # or plan(autotune.best_tile_config(b))
    b.launch()          # or b.graph_launch(stream)
"""
from __future__ import annotations

import ctypes

import torch

from . import abi
from .image import Image


def tile_configs():
    """[(k_outputs, warps, threads)] of the work-item configurations: target
    outputs per work item in units of 1024, warps and threads per CTA."""
    lib = abi.load()
    out = []
    for i in range(lib.ndlgpu_batch_tile_configs()):
        tx, ty, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        abi.check(lib.ndlgpu_batch_tile_config_info(i, ctypes.byref(tx), ctypes.byref(ty), ctypes.byref(nt)))
        out.append((tx.value, ty.value, nt.value))
    return out


class Batch:
    def __init__(self):
        self._lib = abi.load()
        h = ctypes.c_void_p()
        abi.check(self._lib.ndlgpu_batch_create(ctypes.byref(h)))
        self._h = h
        self._keep = []          # the Images stay alive while the batch exists
        self.signature = []      # (rank, extents, taps per pass, border, adjoint) per instance
        self.tile_config = None

    def add(self, src: Image, dst: Image, passes, border, adjoint=False):
        arr, keep = abi.make_passes(passes)
        sv, dv = src.abi_view(), dst.abi_view()
        abi.check(self._lib.ndlgpu_batch_add(self._h, ctypes.byref(sv), ctypes.byref(dv), len(arr), arr, int(border),
                                             1 if adjoint else 0))
        self._keep += [src, dst]
        self.signature.append((src.dim, tuple(src.extent()), tuple(len(p[1]) for p in passes), int(border),
                               bool(adjoint), str(src.dtype)))

    def plan(self, tile_config=-1):
        abi.check(self._lib.ndlgpu_batch_plan(self._h, int(tile_config)))
        self.tile_config = tile_config

    def launch(self, stream=None):
        s = (stream or torch.cuda.current_stream()).cuda_stream
        abi.check(self._lib.ndlgpu_batch_launch(self._h, ctypes.c_void_p(s)))

    def graph_launch(self, stream=None):
        """Replays the launch from a CUDA graph (captured on first use; the
        stream must not be the legacy default stream)."""
        s = (stream or torch.cuda.current_stream()).cuda_stream
        abi.check(self._lib.ndlgpu_batch_graph_launch(self._h, ctypes.c_void_p(s)))

    def info(self):
        n, it, el = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
        abi.check(self._lib.ndlgpu_batch_info(self._h, ctypes.byref(n), ctypes.byref(it), ctypes.byref(el)))
        return {"instances": n.value, "items": it.value, "elements": el.value}

    def close(self):
        if self._h:
            self._lib.ndlgpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
