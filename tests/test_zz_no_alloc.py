"""cn_euler_rk3_stage_noalloc (fixed device scratch, no allocation) against
cn_euler_rk3_stage (cudaMalloc'd scratch), both called through the C ABI.

Two calls in a row (stage 1, then stage 2 reading stage 1's output) must give
the same fields bit for bit and the same conservation sums within 1e-12
relative; a grid above the fixed scratch's limit is rejected."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GAMMA = 1.4
SUM_RTOL = 1e-12
_P, _I, _D = C.c_void_p, C.c_int, C.c_double


def _abi():
    from cubismnova_b200 import _lib
    lib = _lib.lib()
    for name in ("cn_euler_rk3_stage", "cn_euler_rk3_stage_noalloc"):
        f = getattr(lib, name)
        f.restype = _I
        f.argtypes = [_P, _P, _P, _P, _I, _D, _D, C.POINTER(C.c_double), _P]
    return lib


def _host(U):
    return np.stack([U.download(c) for c in range(5)])


def _stage(lib, name, bcsrc, Us, Un, out, stage, dt):
    sums = (C.c_double * 5)()
    rc = getattr(lib, name)(bcsrc.handle, Us.handle, Un.handle if Un is not None else None, out.handle, stage,
                            dt, GAMMA, sums, None)
    assert rc == 0, lib.cn_last_error_string().decode()
    return np.array(list(sums))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_stage_matches_allocating_stage(cn, dtype):
    import torch
    lib = _abi()
    nb, n = (2, 2, 2), (16, 16, 16)
    U = cn.Grid.Cartesian(nb, n, ncomp=5, dtype=dtype)
    cn.workloads.euler_pulse(U, seed=11)
    cn.workloads.euler_bcs(U)
    a1, a2, b1, b2 = (cn.euler.like(U) for _ in range(4))
    dt = cn.euler.cfl_dt(U, 0.3)
    # call 1: stage 1; call 2: stage 2 on call 1's output
    s_ref1 = _stage(lib, "cn_euler_rk3_stage", U, U, None, a1, 1, dt)
    s_ref2 = _stage(lib, "cn_euler_rk3_stage", U, a1, U, a2, 2, dt)
    s_new1 = _stage(lib, "cn_euler_rk3_stage_noalloc", U, U, None, b1, 1, dt)
    s_new2 = _stage(lib, "cn_euler_rk3_stage_noalloc", U, b1, U, b2, 2, dt)
    torch.cuda.synchronize()
    assert np.array_equal(_host(b1), _host(a1))
    assert np.array_equal(_host(b2), _host(a2))
    for got, want in ((s_new1, s_ref1), (s_new2, s_ref2)):
        assert np.all(np.abs(got - want) <= SUM_RTOL * np.maximum(1.0, np.abs(want))), (got, want)
    # the sums are those of the stage output
    vol = float(np.prod(U.getCellSize()))
    host2 = _host(b2)
    for c in range(5):
        ref = float(np.sum(U.blocks_view(host2[c]).astype(np.float64))) * vol
        assert abs(s_new2[c] - ref) <= SUM_RTOL * max(1.0, abs(ref))


def test_noalloc_stage_rejects_grid_above_limit(cn):
    lib = _abi()
    # 513 blocks of 32^3 cells = 32832 tiles of 8^3 > 32768
    U = cn.Grid.Cartesian((513, 1, 1), (32, 32, 32), ncomp=5, dtype=np.float32)
    sums = (C.c_double * 5)()
    rc = lib.cn_euler_rk3_stage_noalloc(U.handle, U.handle, None, U.handle, 1, 1e-3, GAMMA, sums, None)
    assert rc == 12  # CN_ERR_UNSUPPORTED
    assert "32768" in lib.cn_last_error_string().decode()
    rc = lib.cn_euler_rk3_stage_noalloc(U.handle, U.handle, None, U.handle, 1, 1e-3, GAMMA, None, None)
    assert rc == 1  # CN_ERR_INVALID_ARGUMENT: sums_out is required
