"""ctypes binding of libcubismnova_b200.so (the C ABI in include/cubismnova_b200.h).

The shared library is built in-tree by ``make -C cubismnova_b200``; if it is
missing it is built on first use (nvcc is required).  There is no CPU
fallback: every compute entry point runs on the GPU and raises if the
library or the device is unavailable.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcubismnova_b200.so")

CN_FLOAT32, CN_FLOAT64, CN_INT32 = 0, 1, 2

_lock = threading.Lock()
_lib = None


class CnStencil(C.Structure):
    _fields_ = [("begin", C.c_int * 3), ("end", C.c_int * 3), ("tensorial", C.c_int)]


def build(force: bool = False) -> str:
    """Compile the library for sm_100a (make -C cubismnova_b200)."""
    args = ["make", "-C", _HERE, "-j8"]
    if force:
        subprocess.run(["make", "-C", _HERE, "clean"], check=True, capture_output=True)
    out = subprocess.run(args, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("building libcubismnova_b200.so failed:\n" + out.stdout + out.stderr)
    return LIB_PATH


# name -> (restype, argtypes)
_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_I3 = C.POINTER(C.c_int)
_D3 = C.POINTER(C.c_double)
_ST = C.POINTER(CnStencil)
_SIGS = {
    "cn_status_string": (C.c_char_p, [_I]),
    "cn_last_error_string": (C.c_char_p, []),
    "cn_abi_version": (_I, []),
    "cn_stencil_check": (_I, [_ST]),
    "cn_grid_create": (_I, [_I3, _I3, _I, _I, _D3, _D3, C.POINTER(_P)]),
    "cn_grid_create_entity": (_I, [_I3, _I3, _I, _I, _I, _D3, _D3, C.POINTER(_P)]),
    "cn_grid_entity": (_I, [_P, C.POINTER(_I), _I3]),
    "cn_grid_destroy": (_I, [_P]),
    "cn_grid_layout": (_I, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_size_t)]),
    "cn_grid_cell_size": (_I, [_P, _D3]),
    "cn_grid_device_error": (_I, [_P, C.POINTER(C.c_int), _I]),
    "cn_debug_wait_timeout": (_I, [_P, _I, _P]),
    "cn_grid_shape": (_I, [_P, _I3]),
    "cn_grid_data": (_I, [_P, _I, C.POINTER(_P)]),
    "cn_grid_upload": (_I, [_P, _I, _P, C.c_size_t, _P]),
    "cn_grid_download": (_I, [_P, _I, _P, C.c_size_t, _P]),
    "cn_grid_to_aos": (_I, [_P, _I, _I, _I3, _I3, _I, _P, _P]),
    "cn_grid_from_aos": (_I, [_P, _I, _I, _I3, _I3, _I, _P, _P]),
    "cn_grid_copy": (_I, [_P, _P, _P]),
    "cn_bc_push": (_I, [_P, _I, _I, _I, _I, _I, _D]),
    "cn_bc_push_boundary": (_I, [_P, _I, _I, _I, _I, _D]),
    "cn_bc_clear": (_I, [_P, _I, _I]),
    "cn_bc_count": (_I, [_P, _I, _I, C.POINTER(_I)]),
    "cn_bc_sync": (_I, [_P, _P]),
    "cn_lab_extent": (_I, [_P, _ST, _I3]),
    "cn_lab_fill": (_I, [_P, _I, _ST, _I, _I, _I, _P, _P]),
    "cn_laplacian": (_I, [_P, _I, _P, _I, _P]),
    "cn_gradient": (_I, [_P, _I, _P, _I, _P]),
    "cn_lap_grad": (_I, [_P, _I, _P, _I, _P, _I, _P]),
    "cn_divergence": (_I, [_P, _I, _P, _I, _P]),
    "cn_ddx_f64": (None, [_I, _I, _I, _P, _I, _I, _P, _I, _I, _D]),
    "cn_ddx_f32": (None, [_I, _I, _I, _P, _I, _I, _P, _I, _I, C.c_float]),
    "cn_ddx_async": (_I, [_I, _I, _I, _I, _P, _I, _I, _P, _I, _I, _D, _P]),
    "cn_calib_fma_peak": (_I, [_I, C.POINTER(C.c_double)]),
    "cn_grid_write_hdf": (_I, [_P, C.c_char_p, C.c_char_p, _I, _I, _I3, _I3, _I, _D, _I, _P]),
    "cn_grid_read_hdf": (_I, [_P, C.c_char_p, _I, _I, _I3, _I3, _I, _P]),
    "cn_h5_write": (_I, [C.c_char_p, C.c_char_p, _I, C.POINTER(C.c_longlong), _I, _P, _I]),
    "cn_h5_query": (_I, [C.c_char_p, C.c_char_p, C.POINTER(_I), C.POINTER(C.c_longlong), C.POINTER(_I)]),
    "cn_h5_read": (_I, [C.c_char_p, C.c_char_p, _I, C.POINTER(C.c_longlong), _I, _P]),
    "cn_xdmf_write": (_I, [C.c_char_p, C.c_char_p, _I, _I3, _I3, _D3, _D3, _I, _I, _D, _I]),
}


def _bind(lib, sigs):
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


_EXTRA_SIGS = []


def register(sigs: dict) -> None:
    """Adds signatures of further entry points (used by submodules)."""
    _EXTRA_SIGS.append(sigs)
    if _lib is not None:
        _bind(_lib, sigs)


def lib():
    """Loads (building first if needed) the C-ABI library."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            _lib = C.CDLL(LIB_PATH)
            _bind(_lib, _SIGS)
            for s in _EXTRA_SIGS:
                _bind(_lib, s)
    return _lib


class CnError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int) -> None:
    if status != 0:
        msg = lib().cn_last_error_string().decode() or lib().cn_status_string(status).decode()
        raise CnError(status, msg)


def ivec3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def dvec3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def stencil_struct(begin, end, tensorial) -> CnStencil:
    s = CnStencil()
    for d in range(3):
        s.begin[d] = int(begin[d])
        s.end[d] = int(end[d])
    s.tensorial = 1 if tensorial else 0
    return s


def fma_peak_tflops(dtype: int) -> float:
    """Measured FMA throughput of the current device (CN_FLOAT64 / CN_FLOAT32)."""
    v = C.c_double()
    check(lib().cn_calib_fma_peak(dtype, C.byref(v)))
    return v.value
