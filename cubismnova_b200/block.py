"""Block::FieldLab on the device (include/Cubism/Block/FieldLab.h).

A lab holds one block's data plus ghost cells for a stencil; here its storage
is a device tensor holding the dense active lab range, filled by the
``cn_lab_fill`` kernel (inner copy, periodic neighbour gather and BCs in the
reference's order and precedence).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .core import IndexRange, Stencil
from .grid import Cartesian, _stream_handle


class BlockBytes:
    def __init__(self, allocated=0, used=0):
        self.allocated, self.used = allocated, used


class FieldLab:
    def __init__(self):
        self._alloc = False
        self._stencil = Stencil(0, 1)
        self._max_range = IndexRange(0)
        self._field = None
        self._range = IndexRange(0)
        self._buf = None

    # Block/FieldLab.h:104-165
    def allocate(self, s: Stencil, max_request_range: IndexRange, force: bool = False):
        import torch
        self._stencil = s
        ext = tuple(e + 2 for e in max_request_range.getExtent())
        self._max_range = IndexRange(ext)
        lab_ext = tuple(ext[d] - s.getBegin()[d] + s.getEnd()[d] - 1 for d in range(3))
        need = lab_ext[0] * lab_ext[1] * lab_ext[2]
        if force or self._buf is None or self._buf.numel() < need:
            self._dtype_hint = None
            self._need = need
            self._buf = None  # allocated on first load, when the dtype is known
        self._alloc = True
        self._torch = torch

    def isAllocated(self):
        return self._alloc

    def getMaximumRange(self):
        return self._max_range

    # Block/FieldLab.h:180-248
    def loadData(self, fid, grid: Cartesian, apply_bc: bool = True, extern_bc=None, comp: int = 0,
                 stream=None):
        if not self._alloc:
            raise RuntimeError("FieldLab: can not load lab data when not allocated first")
        flat = grid.flat_index(fid)
        ext = grid.getBlockExtent()
        if any(e > m for e, m in zip(ext, self._max_range.getExtent())):
            raise RuntimeError("FieldLab: block larger than the allocated maximum range")
        torch = self._torch
        tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
               np.dtype(np.int32): torch.int32}[grid.dtype]
        if self._buf is None or self._buf.dtype != tdt or self._buf.numel() < self._need:
            self._buf = torch.zeros(self._need, dtype=tdt, device="cuda")
        saved = None
        if extern_bc is not None:
            vec = grid.field(flat, comp).getBC()
            saved = list(vec)
            vec.clear()
            for b in extern_bc:
                vec.push_back(b)
        try:
            st = self._stencil.as_struct()
            _lib.check(_lib.lib().cn_lab_fill(grid.handle, comp, C.byref(st), flat, 1,
                                              1 if apply_bc else 0,
                                              C.c_void_p(self._buf.data_ptr()),
                                              _stream_handle(stream)))
        finally:
            if saved is not None:
                vec = grid.field(flat, comp).getBC()
                vec.clear()
                for b in saved:
                    vec.push_back(b)
        self._field = grid.field(flat, comp)
        # the device lab has the strides of the grid's largest lab; a node or
        # face block that is not last along a grown direction is one smaller
        self._layout = tuple(ext[d] - self._stencil.getBegin()[d] + self._stencil.getEnd()[d] - 1
                             for d in range(3))
        self._range = IndexRange(grid.block_extent(flat))

    def getActiveStencil(self):
        return self._stencil

    def getActiveRange(self):
        return self._range

    def getActiveLabRange(self):
        b = self._stencil.getBegin()
        e = tuple(self._range.getExtent()[d] + self._stencil.getEnd()[d] - 1 for d in range(3))
        return IndexRange(b, e)

    def getActiveField(self):
        if self._field is None:
            raise RuntimeError("FieldLab: no field loaded")
        return self._field

    def getMemoryFootprint(self):
        if not self._alloc or self._buf is None:
            return BlockBytes()
        used = self.getActiveLabRange().size() * self._buf.element_size()
        return BlockBytes(self._buf.numel() * self._buf.element_size(), used)

    @property
    def data(self):
        """Device tensor (Lz, Ly, Lx) of the active lab range (a view with the
        strides of the grid's largest lab)."""
        lr = self.getActiveLabRange().getExtent()
        L = self._layout
        n = L[0] * L[1] * L[2]
        return self._buf[:n].view(L[2], L[1], L[0])[: lr[2], : lr[1], : lr[0]]

    def numpy(self):
        return self.data.cpu().numpy()

    def __getitem__(self, p):
        b = self._stencil.getBegin()
        return self.data[p[2] - b[2], p[1] - b[1], p[0] - b[0]].item()
