"""Compressible Euler on a device grid: fused lab + WENO5-JS + Rusanov flux
divergence, SSP-RK3 stages, conservation sums and CFL speeds (csrc/euler.cu).

A state is a ``Grid.Cartesian`` with 5 components (rho, rho*u, rho*v, rho*w, E);
BCs are taken per component from the grid's BC vectors (as in
``FieldLab::loadData``), so a component can be, e.g., Dirichlet in z with its
own far-field value.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .grid import Cartesian, _stream_handle

_P, _I, _D = C.c_void_p, C.c_int, C.c_double
_lib.register({
    "cn_euler_rhs": (_I, [_P, _I, _D, _P, _I, _P]),
    "cn_euler_rk3_stage": (_I, [_P, _P, _P, _P, _I, _D, _D, C.POINTER(C.c_double), _P]),
    "cn_euler_rk3_step": (_I, [_P, _P, _P, _D, _D, C.POINTER(C.c_double), _P]),
    "cn_euler_max_speed": (_I, [_P, _D, C.POINTER(C.c_double), _P]),
})

GAMMA = 1.4


def rhs(U: Cartesian, out: Cartesian, gamma: float = GAMMA, stream=None):
    """out[0:5] = L(U) = -div F(U)."""
    _lib.check(_lib.lib().cn_euler_rhs(U.handle, 0, gamma, out.handle, 0, _stream_handle(stream)))


def rk3_stage(bcsrc: Cartesian, Us: Cartesian, Un, out: Cartesian, stage: int, dt: float,
              gamma: float = GAMMA, want_sums: bool = False, stream=None):
    sums = (C.c_double * 5)() if want_sums else None
    _lib.check(_lib.lib().cn_euler_rk3_stage(bcsrc.handle, Us.handle, Un.handle if Un is not None else None,
                                             out.handle, stage, dt, gamma, sums, _stream_handle(stream)))
    return list(sums) if want_sums else None


def rk3_step(U: Cartesian, work1: Cartesian, work2: Cartesian, dt: float, gamma: float = GAMMA,
             want_sums: bool = False, stream=None):
    """U <- U^{n+1} (three fused stage kernels).  With want_sums the FP64
    integrals of the 5 conserved variables of U^{n+1} are returned."""
    sums = (C.c_double * 5)() if want_sums else None
    _lib.check(_lib.lib().cn_euler_rk3_step(U.handle, work1.handle, work2.handle, dt, gamma, sums,
                                            _stream_handle(stream)))
    return list(sums) if want_sums else None


def max_speed(U: Cartesian, gamma: float = GAMMA, stream=None):
    out = (C.c_double * 3)()
    _lib.check(_lib.lib().cn_euler_max_speed(U.handle, gamma, out, _stream_handle(stream)))
    return tuple(out)


def cfl_dt(U: Cartesian, cfl: float = 0.3, gamma: float = GAMMA, stream=None) -> float:
    """dt = cfl / sum_d (max(|u_d|+c) / h_d)."""
    s = max_speed(U, gamma, stream)
    h = U.getCellSize()
    return cfl / sum(s[d] / h[d] for d in range(3))


def like(U: Cartesian) -> Cartesian:
    """A work grid of the same geometry (blocks, cells and physical extent)
    and dtype (no BCs)."""
    nb, n = U.getSize(), U.getBlockCells()
    begin = getattr(U, "_begin", None)
    end = getattr(U, "_end", None)
    if begin is None or end is None:  # a view of a library-made grid: its extent from the cell size
        begin = (0.0, 0.0, 0.0)
        h = U.getCellSize()
        end = tuple(nb[d] * n[d] * h[d] for d in range(3))
    return Cartesian(nb, n, begin, end, ncomp=5, dtype=U.dtype)
