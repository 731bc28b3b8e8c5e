"""Fused lab + stencil operators (one kernel each, grids resident on the GPU).

Each operator loads every block's lab (stencil (-1,2), BCs of the input
component) and applies the stencil in the same kernel; see
``cubismnova_b200/csrc/fd.cu``.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .grid import Cartesian, _stream_handle


def laplacian(u: Cartesian, out: Cartesian, comp: int = 0, out_comp: int = 0, stream=None):
    """7-point Laplacian (Kernel/Laplacian/Laplacian.cpp:123-130 grouping)."""
    _lib.check(_lib.lib().cn_laplacian(u.handle, comp, out.handle, out_comp, _stream_handle(stream)))


def gradient(u: Cartesian, out: Cartesian, comp: int = 0, out_comp: int = 0, stream=None):
    """Central gradient into out components out_comp..out_comp+2."""
    _lib.check(_lib.lib().cn_gradient(u.handle, comp, out.handle, out_comp, _stream_handle(stream)))


def lap_grad(u: Cartesian, lap: Cartesian, grad: Cartesian, comp: int = 0, lap_comp: int = 0,
             grad_comp: int = 0, stream=None):
    """Laplacian and gradient from one lab load."""
    _lib.check(_lib.lib().cn_lap_grad(u.handle, comp, lap.handle, lap_comp, grad.handle, grad_comp,
                                      _stream_handle(stream)))


def divergence(v: Cartesian, out: Cartesian, comp: int = 0, out_comp: int = 0, stream=None):
    """Divergence of components comp..comp+2 (nova.cpp:113-126)."""
    _lib.check(_lib.lib().cn_divergence(v.handle, comp, out.handle, out_comp, _stream_handle(stream)))


def load_labs(u: Cartesian, stencil, out=None, comp: int = 0, block_begin: int = 0, count: int = None,
              apply_bc: bool = True, stream=None):
    """Cartesian::loadLab for a range of blocks in one launch (the block loop
    of Grid/Cartesian.h:412-427 over FieldLab::loadData, Block/FieldLab.h:180-224):
    the labs of blocks [block_begin, block_begin + count) of component
    ``comp`` for ``stencil`` (a Core.Stencil) into ``out``, a CUDA tensor of
    count x (E2, E1, E0) values (x fastest; cells the reference leaves
    undefined keep out's values).  Returns out."""
    import torch
    st = stencil.as_struct()
    ext = (C.c_int * 3)()
    _lib.check(_lib.lib().cn_lab_extent(u.handle, C.byref(st), ext))
    n = u.getSize()[0] * u.getSize()[1] * u.getSize()[2]
    count = n - block_begin if count is None else count
    shape = (count, ext[2], ext[1], ext[0])
    tdt = {4: torch.float32, 8: torch.float64}[u.dtype.itemsize] if u.dtype.kind == "f" else torch.int32
    if out is None:
        out = torch.zeros(shape, dtype=tdt, device="cuda")
    elif tuple(out.shape) != shape or out.dtype != tdt or not out.is_contiguous() or not out.is_cuda:
        raise ValueError(f"load_labs: out must be a contiguous CUDA {tdt} tensor of shape {shape}")
    _lib.check(_lib.lib().cn_lab_fill(u.handle, comp, C.byref(st), int(block_begin), int(count),
                                      1 if apply_bc else 0, C.c_void_p(out.data_ptr()), _stream_handle(stream)))
    return out


def ddx(src_ptr: int, dst_ptr: int, extent, src_pitch, dst_pitch, factor: float, dtype="f64",
        stream=None):
    """The ISPC benchmark kernel ABI (BaseBenchmark.h:27-37) on device pointers.

    ``src_ptr`` points at the first inner element of a pitched lab;
    pitches are (x_pitch, xy_pitch) in elements."""
    dt = _lib.CN_FLOAT64 if dtype in ("f64", "float64") else _lib.CN_FLOAT32
    _lib.check(_lib.lib().cn_ddx_async(dt, int(extent[0]), int(extent[1]), int(extent[2]),
                                       C.c_void_p(src_ptr), int(src_pitch[0]), int(src_pitch[1]),
                                       C.c_void_p(dst_ptr), int(dst_pitch[0]), int(dst_pitch[1]),
                                       C.c_double(factor), _stream_handle(stream)))
