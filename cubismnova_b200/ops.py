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
