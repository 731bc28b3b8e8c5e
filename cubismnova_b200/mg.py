"""Geometric multigrid for div(k grad p) = f on a periodic device grid
(csrc/mg.cu): FP32 V-cycles with weighted Jacobi, FP64 coarsest solve and an
FP64 defect-correction outer loop with FP64 residual norms."""
from __future__ import annotations

import ctypes as C

from . import _lib
from .grid import Cartesian, _stream_handle

_P, _I, _D = C.c_void_p, C.c_int, C.c_double
_PD = C.POINTER(C.c_double)
_lib.register({
    "cn_mg_create": (_I, [_P, _I, _I, _D, _I, C.POINTER(_P)]),
    "cn_mg_destroy": (_I, [_P]),
    "cn_mg_levels": (_I, [_P, C.POINTER(_I), C.POINTER(_I)]),
    "cn_mg_vcycle": (_I, [_P, _P, _P, _P]),
    "cn_mg_residual": (_I, [_P, _P, _P, _P, _PD, _PD, _P]),
    "cn_mg_solve": (_I, [_P, _P, _P, _D, _I, C.POINTER(_I), _PD, _P]),
    "cn_mg_jacobi": (_I, [_P, _P, _P, _P, _P]),
    "cn_mg_restrict_residual": (_I, [_P, _P, _P, _P, _P]),
    "cn_mg_prolong": (_I, [_P, _P, _P, _P]),
    "cn_mg_level_grid": (_I, [_P, _I, _I, C.POINTER(_P)]),
})


class Multigrid:
    def __init__(self, k: Cartesian, nu1: int = 2, nu2: int = 2, omega: float = 0.8,
                 max_levels: int = 0):
        h = C.c_void_p()
        _lib.check(_lib.lib().cn_mg_create(k.handle, nu1, nu2, omega, max_levels, C.byref(h)))
        self._h, self.k = h, k
        nl, cc = C.c_int(), C.c_int()
        _lib.check(_lib.lib().cn_mg_levels(h, C.byref(nl), C.byref(cc)))
        self.nlevels, self.coarsest_cells = nl.value, cc.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().cn_mg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def level(self, l: int, which: str = "p") -> Cartesian:
        g = C.c_void_p()
        _lib.check(_lib.lib().cn_mg_level_grid(self._h, l, {"p": 0, "f": 1, "k": 2}[which], C.byref(g)))
        return Cartesian.view_of(g, owner=self)

    def vcycle(self, rhs: Cartesian, e: Cartesian, stream=None):
        _lib.check(_lib.lib().cn_mg_vcycle(self._h, rhs.handle, e.handle, _stream_handle(stream)))

    def residual(self, p64: Cartesian, f: Cartesian, r32: Cartesian = None, stream=None):
        rr, ff = C.c_double(), C.c_double()
        _lib.check(_lib.lib().cn_mg_residual(self._h, p64.handle, f.handle, r32.handle if r32 else None,
                                             C.byref(rr), C.byref(ff), _stream_handle(stream)))
        return rr.value, ff.value

    def solve(self, f: Cartesian, p64: Cartesian, rtol: float = 1e-8, max_cycles: int = 100, stream=None):
        cyc, rel = C.c_int(), C.c_double()
        _lib.check(_lib.lib().cn_mg_solve(self._h, f.handle, p64.handle, rtol, max_cycles, C.byref(cyc),
                                          C.byref(rel), _stream_handle(stream)))
        return cyc.value, rel.value

    def jacobi(self, pin: Cartesian, f: Cartesian, pout: Cartesian, stream=None):
        _lib.check(_lib.lib().cn_mg_jacobi(self._h, pin.handle, f.handle, pout.handle, _stream_handle(stream)))

    def restrict_residual(self, p: Cartesian, f: Cartesian, fc: Cartesian, stream=None):
        _lib.check(_lib.lib().cn_mg_restrict_residual(self._h, p.handle, f.handle, fc.handle,
                                                      _stream_handle(stream)))

    def prolong(self, ec: Cartesian, p: Cartesian, stream=None):
        _lib.check(_lib.lib().cn_mg_prolong(self._h, ec.handle, p.handle, _stream_handle(stream)))
