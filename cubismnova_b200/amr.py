"""Blocks of uneven sizes on two refinement levels (csrc/amr.cu): layout,
level-interface ghost fill, fused Euler SSP-RK3 stages as persistent launches
over a tile work list, schedule autotuning and CUDA graph capture."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .grid import _stream_handle

_P, _I, _D = C.c_void_p, C.c_int, C.c_double
_I64 = C.c_int64
_lib.register({
    "cn_amr_create": (_I, [_I, _P, _P, _P, _I, _I, _I, C.POINTER(_P)]),
    "cn_amr_create_box": (_I, [_I, _P, _P, _P, C.POINTER(_I), _I, _I, C.POINTER(_P)]),
    "cn_amr_destroy": (_I, [_P]),
    "cn_amr_info": (_I, [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I)]),
    "cn_amr_block_offset": (_I, [_P, _I, C.POINTER(_I64)]),
    "cn_amr_data": (_I, [_P, _I, C.POINTER(_P)]),
    "cn_amr_lab_fill": (_I, [_P, _I, _I, _I, _P, _P]),
    "cn_amr_rk3_stage": (_I, [_P, _P, _P, _I, _D, _D, _P]),
    "cn_amr_rk3_step": (_I, [_P, _P, _P, _D, _D, _P]),
    "cn_amr_set_schedule": (_I, [_P, _I, _I]),
    "cn_amr_set_work_unit": (_I, [_P, _I]),
    "cn_amr_get_schedule": (_I, [_P, C.POINTER(C.c_int)]),
    "cn_amr_set_work_shape": (_I, [_P, C.POINTER(C.c_int)]),
    "cn_amr_get_work_shape": (_I, [_P, C.POINTER(C.c_int)]),
    "cn_amr_autotune": (_I, [_P, _P, _P, _D, _D, _I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_D), _P]),
    "cn_graph_begin": (_I, [_P]),
    "cn_graph_end": (_I, [_P, C.POINTER(_P)]),
    "cn_graph_launch": (_I, [_P, _P]),
    "cn_graph_destroy": (_I, [_P]),
})


class AmrGrid:
    """Blocks (level, cells, origin in level-1 units) tiling a periodic unit box
    of ``fine_extent`` level-1 cells (one extent for a cube, or (Lx, Ly, Lz));
    cells are cubic with h = cell size / Lx; ``ncomp`` components."""

    def __init__(self, levels, cells, origins, fine_extent, ncomp: int = 5, dtype=np.float64):
        self.levels = np.asarray(levels, dtype=np.int32)
        self.cells = np.asarray(cells, dtype=np.int32)
        self.origins = np.ascontiguousarray(np.asarray(origins, dtype=np.int32).reshape(-1, 3))
        ext = np.broadcast_to(np.asarray(fine_extent, dtype=np.int64), (3,))
        self.L = tuple(int(e) for e in ext)
        self.L1 = self.L[0]
        self.ncomp, self.dtype = int(ncomp), np.dtype(dtype)
        dt = {np.dtype(np.float32): _lib.CN_FLOAT32, np.dtype(np.float64): _lib.CN_FLOAT64}[self.dtype]
        h = C.c_void_p()
        _lib.check(_lib.lib().cn_amr_create_box(len(self.levels), self.levels.ctypes.data_as(C.c_void_p),
                                                self.cells.ctypes.data_as(C.c_void_p),
                                                self.origins.ctypes.data_as(C.c_void_p), _lib.ivec3(self.L),
                                                self.ncomp, dt, C.byref(h)))
        self._h = h
        tc, cs, ni = C.c_int64(), C.c_int64(), C.c_int()
        _lib.check(_lib.lib().cn_amr_info(h, C.byref(tc), C.byref(cs), C.byref(ni)))
        self.total_cells, self.comp_stride, self.nitems = tc.value, cs.value, ni.value
        self.offsets = np.concatenate([[0], np.cumsum(self.cells.astype(np.int64) ** 3)])[:-1]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().cn_amr_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def nblocks(self):
        return len(self.levels)

    def like(self):
        return AmrGrid(self.levels, self.cells, self.origins, self.L, self.ncomp, self.dtype)

    def tensor(self, comp=0):
        import torch
        p = C.c_void_p()
        _lib.check(_lib.lib().cn_amr_data(self._h, comp, C.byref(p)))
        typ = {np.dtype(np.float32): "<f4", np.dtype(np.float64): "<f8"}[self.dtype]

        class _CAI:
            __cuda_array_interface__ = {"shape": (self.comp_stride,), "typestr": typ, "data": (p.value, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_CAI(), device="cuda")

    def download(self, comp=0):
        return self.tensor(comp).cpu().numpy()

    def upload(self, arr, comp=0):
        import torch
        self.tensor(comp).copy_(torch.as_tensor(np.ascontiguousarray(arr, dtype=self.dtype)))

    def lab(self, comp: int, ghost: int, block: int, fill=0.0):
        import torch
        n = int(self.cells[block])
        E = n + 2 * ghost
        tdt = torch.float64 if self.dtype == np.float64 else torch.float32
        buf = torch.full((E, E, E), fill, dtype=tdt, device="cuda")
        _lib.check(_lib.lib().cn_amr_lab_fill(self._h, comp, ghost, block, C.c_void_p(buf.data_ptr()),
                                              _stream_handle(None)))
        return buf

    def set_schedule(self, order: int, ctas: int, unit: int = None, shape=None):
        """Work-list order, persistent grid size and (optionally) the CTA's
        work tile: ``shape`` = 8^3 tiles along (x, y, z), each 1, 2 or 4, or
        ``unit`` = t for the shape (t, 1, 1)."""
        if unit is not None:
            _lib.check(_lib.lib().cn_amr_set_work_unit(self._h, unit))
        if shape is not None:
            _lib.check(_lib.lib().cn_amr_set_work_shape(self._h, (C.c_int * 3)(*[int(v) for v in shape])))
        _lib.check(_lib.lib().cn_amr_set_schedule(self._h, order, ctas))

    def schedule(self):
        """(order, ctas, tiles per work tile) of this layout."""
        out = (C.c_int * 3)()
        _lib.check(_lib.lib().cn_amr_get_schedule(self._h, out))
        return tuple(out)

    def work_shape(self):
        """The CTA's work tile in 8^3 tiles along (x, y, z)."""
        out = (C.c_int * 3)()
        _lib.check(_lib.lib().cn_amr_get_work_shape(self._h, out))
        return tuple(out)

    def box(self):
        """Physical extents of the periodic box: (1, Ly/Lx, Lz/Lx)."""
        return tuple(e / self.L[0] for e in self.L)

    def cell_centres(self):
        """(x, y, z) cell-centre coordinates of all cells, block order (torch,
        cuda), in the box [0,1] x [0, Ly/Lx] x [0, Lz/Lx]."""
        import torch
        dev = "cuda"
        n = torch.tensor(self.cells, device=dev, dtype=torch.int64)
        ncell = n ** 3
        blk = torch.repeat_interleave(torch.arange(self.nblocks, device=dev), ncell)
        off = torch.tensor(self.offsets, device=dev, dtype=torch.int64)
        loc = torch.arange(self.total_cells, device=dev, dtype=torch.int64) - off[blk]
        nb = n[blk]
        lx, ly, lz = loc % nb, (loc // nb) % nb, loc // (nb * nb)
        cs = torch.where(torch.tensor(self.levels, device=dev)[blk] == 0, 2.0, 1.0).to(torch.float64)
        org = torch.tensor(self.origins, device=dev, dtype=torch.float64)[blk]
        x = (org[:, 0] + (lx.to(torch.float64) + 0.5) * cs) / self.L1
        y = (org[:, 1] + (ly.to(torch.float64) + 0.5) * cs) / self.L1
        z = (org[:, 2] + (lz.to(torch.float64) + 0.5) * cs) / self.L1
        return x, y, z


def rk3_stage(Us: AmrGrid, Un, out: AmrGrid, stage: int, dt: float, gamma: float = 1.4, stream=None):
    _lib.check(_lib.lib().cn_amr_rk3_stage(Us.handle, Un.handle if Un is not None else None, out.handle, stage,
                                           dt, gamma, _stream_handle(stream)))


def rk3_step(U: AmrGrid, w1: AmrGrid, w2: AmrGrid, dt: float, gamma: float = 1.4, stream=None):
    _lib.check(_lib.lib().cn_amr_rk3_step(U.handle, w1.handle, w2.handle, dt, gamma, _stream_handle(stream)))


def autotune(U: AmrGrid, w1: AmrGrid, w2: AmrGrid, dt: float, gamma: float = 1.4, reps: int = 2, stream=None):
    """Picks the fastest work-list order, work-tile shape and persistent
    grid (advances U); returns (order, ctas, ms), the shape by
    U.work_shape()."""
    o, c, ms = C.c_int(), C.c_int(), C.c_double()
    _lib.check(_lib.lib().cn_amr_autotune(U.handle, w1.handle, w2.handle, dt, gamma, reps, C.byref(o), C.byref(c),
                                          C.byref(ms), _stream_handle(stream)))
    return o.value, c.value, ms.value


class Graph:
    """A captured CUDA graph of library calls issued on one stream."""

    def __init__(self, handle):
        self._h = handle

    @staticmethod
    def capture(fn, stream):
        _lib.check(_lib.lib().cn_graph_begin(_stream_handle(stream)))
        try:
            fn()
        finally:
            h = C.c_void_p()
            _lib.check(_lib.lib().cn_graph_end(_stream_handle(stream), C.byref(h)))
        return Graph(h)

    def launch(self, stream):
        _lib.check(_lib.lib().cn_graph_launch(self._h, _stream_handle(stream)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().cn_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
