"""Image views over device memory, with ndl's view arithmetic.

``Image`` mirrors the non-owning view of ndl's ``Image<T,DIM>``
(image/core.h:50-972): a base pointer, an extent and signed element strides in
ndl axis order (axis 0 fastest for a default layout, image/core.h:858-864).
The view builders reproduce the reference's rules exactly:

* ``view(start, end, step)``  -- image/core.h:647-703 (inclusive ends,
  negative indices count from the end, a negative step mirrors and anchors at
  ``end``; extent = _ceil(float(len) / |step|), image/core.h:859-861)
* ``slice(dim, index)``       -- image/core.h:709-712, :814-823
* ``swap_axes(a, b)``         -- image/core.h:717-731
* ``mirror(dim)``             -- image/core.h:735-757

The memory belongs to a torch tensor (kept alive by the view); ``tensor()``
returns a torch view of exactly the elements the Image covers, with torch's
axis order reversed (torch dim 0 = ndl axis DIM-1).
"""
from __future__ import annotations

import math

import torch

from . import abi

TORCH_DTYPE = {
    torch.uint8: abi.U8, torch.int8: abi.I8, torch.int16: abi.I16, torch.int32: abi.I32,
    torch.int64: abi.I64, torch.float32: abi.F32, torch.float64: abi.F64, torch.float16: abi.F16,
    torch.bfloat16: abi.BF16,
}
for _name, _code in (("uint16", abi.U16), ("uint32", abi.U32), ("uint64", abi.U64)):
    if hasattr(torch, _name):
        TORCH_DTYPE[getattr(torch, _name)] = _code


def _ceil(num):
    """_ceil of mathHelpers.h:17 (truncate, bump positive non-integers)."""
    t = int(num)
    return t if float(t) == num else t + (1 if num > 0 else 0)


def _f32(x):
    """The value of a C++ float computed from a double (round to nearest)."""
    import struct
    return struct.unpack("f", struct.pack("f", x))[0]


class BorderMode:
    """ndl::BorderMode (image/border_mode.h:14-19)."""
    Clamp = abi.CLAMP
    Wrap = abi.WRAP
    Reflect = abi.REFLECT


class Image:
    """Non-owning strided view of device memory held by a torch tensor."""

    def __init__(self, storage: torch.Tensor, offset: int, extent, stride):
        if storage.dim() != 1 or not storage.is_contiguous():
            storage = storage.reshape(-1) if storage.is_contiguous() else storage
        self._storage = storage          # 1-D tensor that owns the memory
        self._offset = int(offset)       # element offset of at({0,..,0})
        self._extent = [int(e) for e in extent]
        self._stride = [int(s) for s in stride]
        if storage.dtype not in TORCH_DTYPE:
            raise TypeError("unsupported element type %s" % storage.dtype)

    # -- construction -----------------------------------------------------
    @classmethod
    def from_tensor(cls, t: torch.Tensor):
        """ndl view of a torch tensor of shape (n_{D-1}, ..., n_0): ndl axis
        i is torch dim D-1-i; any torch strides are kept."""
        if t.dim() < 1 or t.dim() > abi.MAX_RANK:
            raise ValueError("rank must be 1..8")
        base = t.as_strided((t.untyped_storage().nbytes() // t.element_size(),), (1,), 0)
        return cls(base, t.storage_offset(), list(t.shape[::-1]), list(t.stride()[::-1]))

    @classmethod
    def empty(cls, extent, dtype=torch.float32, device="cuda"):
        """A contiguous image of the given ndl extent (axis 0 fastest),
        like OwnedImage (image/owned.h:100-102) but uninitialised."""
        n = 1
        for e in extent:
            n *= int(e)
        buf = torch.empty(n, dtype=dtype, device=device)
        return cls(buf, 0, extent, _default_strides(extent))

    @classmethod
    def zeros(cls, extent, dtype=torch.float32, device="cuda"):
        img = cls.empty(extent, dtype, device)
        img._storage.zero_()
        return img

    # -- the minimal interface -------------------------------------------
    def extent(self):
        return list(self._extent)

    def stride(self):
        return list(self._stride)

    @property
    def dim(self):
        return len(self._extent)

    @property
    def dtype(self):
        return self._storage.dtype

    @property
    def device(self):
        return self._storage.device

    def size(self):
        n = 1
        for e in self._extent:
            n *= e
        return n

    def data_ptr(self):
        return self._storage.data_ptr() + self._offset * self._storage.element_size()

    def abi_view(self):
        return abi.make_view(self.data_ptr(), TORCH_DTYPE[self.dtype], self._extent, self._stride)

    def tensor(self):
        """torch view of the covered elements, shape (n_{D-1}, ..., n_0)."""
        # torch.as_strided rejects negative strides: build the positive-stride
        # view, then flip the mirrored dims.
        off = self._offset
        shape, strides, flips = [], [], []
        for d, (e, s) in enumerate(zip(self._extent[::-1], self._stride[::-1])):
            if s < 0:
                off += (e - 1) * s
                s = -s
                flips.append(d)
            shape.append(e)
            strides.append(s)
        t = self._storage.as_strided(shape, strides, off)
        return t.flip(flips) if flips else t

    # -- view builders (image/core.h:647-757) -----------------------------
    def view(self, start=(), end=(), step=()):
        start, end, step = list(start), list(end), list(step)
        off = self._offset
        ext, st = [], []
        for i in range(self.dim):
            s = start[i] if i < len(start) else 0
            e = end[i] if i < len(end) else -1
            sp = step[i] if i < len(step) else 1
            if sp == 0:
                raise IndexError("Image::view: step must not be 0 (dimension %d)" % i)
            if s < 0:
                s += self._extent[i]
            if e < 0:
                e += self._extent[i]
            if s < 0 or s >= self._extent[i] or e < 0 or e >= self._extent[i] or e < s:
                raise IndexError("Image::view: [start=%d, end=%d] is not a valid range for dimension %d" % (s, e, i))
            o = e if sp < 0 else s
            off += o * self._stride[i]
            ext.append(_ceil(_f32(_f32(float(1 + e - s)) / abs(sp))))
            st.append(self._stride[i] * sp)
        return Image(self._storage, off, ext, st)

    def slice(self, dim, index):
        if self.dim < 2:
            raise ValueError("cannot slice a 1-D image")
        off = self._offset + index * self._stride[dim]
        ext = [e for i, e in enumerate(self._extent) if i != dim]
        st = [s for i, s in enumerate(self._stride) if i != dim]
        return Image(self._storage, off, ext, st)

    def swap_axes(self, a, b):
        ext, st = list(self._extent), list(self._stride)
        ext[a], ext[b] = ext[b], ext[a]
        st[a], st[b] = st[b], st[a]
        return Image(self._storage, self._offset, ext, st)

    def mirror(self, dim):
        st = list(self._stride)
        off = self._offset + (self._extent[dim] - 1) * st[dim]
        st[dim] = -st[dim]
        return Image(self._storage, off, self._extent, st)

    def __repr__(self):
        return "Image(dtype=%s, extent=%s, stride=%s)" % (self.dtype, self._extent, self._stride)


def _default_strides(extent):
    st, m = [], 1
    for e in extent:
        st.append(m)
        m *= int(e)
    return st
