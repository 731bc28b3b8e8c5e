"""cn_euler_rk3_stage_noalloc (fixed device scratch, no allocation) against
cn_euler_rk3_stage (cudaMalloc'd scratch), both called through the C ABI.

The no-allocation stage is for hosts that cannot call cudaMalloc while they
run: a solver whose device memory is reserved up front by another allocator,
or one that must not let a first-time cudaMalloc/cudaFree synchronise the
device mid-run.  Both entry points run the same stage and reduction kernels in
the same order, so two calls in a row (stage 1, then stage 2 reading stage 1's
output) must give the same fields and the same conservation sums bit for bit.
A grid at the scratch's limit (32768 tiles of 8^3) runs without changing the
device's free memory; one above it is rejected; BC vectors that grew since
their last upload are refused until cn_bc_sync has run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GAMMA = 1.4
_P, _I, _D = C.c_void_p, C.c_int, C.c_double
CN_ERR_INVALID_ARGUMENT, CN_ERR_UNSUPPORTED = 1, 12


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


def _call(lib, name, bcsrc, Us, Un, out, stage, dt):
    sums = (C.c_double * 5)()
    rc = getattr(lib, name)(bcsrc.handle, Us.handle, Un.handle if Un is not None else None, out.handle, stage,
                            dt, GAMMA, sums, None)
    return rc, np.array(list(sums))


def _stage(lib, name, bcsrc, Us, Un, out, stage, dt):
    rc, sums = _call(lib, name, bcsrc, Us, Un, out, stage, dt)
    assert rc == 0, lib.cn_last_error_string().decode()
    return sums


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
    assert np.array_equal(s_new1, s_ref1)
    assert np.array_equal(s_new2, s_ref2)
    # the sums are those of the stage output
    vol = float(np.prod(U.getCellSize()))
    host2 = _host(b2)
    for c in range(5):
        ref = float(np.sum(U.blocks_view(host2[c]).astype(np.float64))) * vol
        assert abs(s_new2[c] - ref) <= 1e-12 * max(1.0, abs(ref))


def test_noalloc_stage_at_the_limit_allocates_nothing(cn):
    """512 blocks of 32^3 = 32768 tiles, the largest grid the scratch holds:
    the device's free memory is the same before and after two calls, and the
    results equal the allocating stage's."""
    import torch
    lib = _abi()
    nb, n = (8, 8, 8), (32, 32, 32)
    U = cn.Grid.Cartesian(nb, n, ncomp=5, dtype=np.float32)
    cn.workloads.euler_pulse(U, seed=3)
    cn.workloads.euler_bcs(U)
    U.sync_bcs()
    b1, b2 = cn.euler.like(U), cn.euler.like(U)
    dt = cn.euler.cfl_dt(U, 0.3)
    # warm call on a small grid: loads the kernels and looks the array up
    W = cn.Grid.Cartesian((1, 1, 1), (8, 8, 8), ncomp=5, dtype=np.float32)
    cn.workloads.euler_pulse(W, seed=1)
    _stage(lib, "cn_euler_rk3_stage_noalloc", W, W, None, cn.euler.like(W), 1, 1e-4)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    s1 = _stage(lib, "cn_euler_rk3_stage_noalloc", U, U, None, b1, 1, dt)
    s2 = _stage(lib, "cn_euler_rk3_stage_noalloc", U, b1, U, b2, 2, dt)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    a1, a2 = cn.euler.like(U), cn.euler.like(U)
    r1 = _stage(lib, "cn_euler_rk3_stage", U, U, None, a1, 1, dt)
    r2 = _stage(lib, "cn_euler_rk3_stage", U, a1, U, a2, 2, dt)
    torch.cuda.synchronize()
    assert np.array_equal(s1, r1) and np.array_equal(s2, r2)
    for c in range(5):
        assert torch.equal(b2.tensor(c), a2.tensor(c))


def test_noalloc_stage_refuses_grown_bc_table(cn):
    """BCs pushed after the last upload that need a larger device table are
    refused (the upload would allocate); after cn_bc_sync the call runs and
    equals the allocating stage."""
    import torch
    lib = _abi()
    nb, n = (2, 2, 2), (8, 8, 8)
    U = cn.Grid.Cartesian(nb, n, ncomp=5)
    cn.workloads.euler_pulse(U, seed=5)
    U.sync_bcs()  # empty BC table uploaded: capacity of one entry
    cn.workloads.euler_bcs(U)
    out = cn.euler.like(U)
    rc, _ = _call(lib, "cn_euler_rk3_stage_noalloc", U, U, None, out, 1, 1e-4)
    assert rc == CN_ERR_INVALID_ARGUMENT
    assert "cn_bc_sync" in lib.cn_last_error_string().decode()
    U.sync_bcs()
    s = _stage(lib, "cn_euler_rk3_stage_noalloc", U, U, None, out, 1, 1e-4)
    ref = cn.euler.like(U)
    r = _stage(lib, "cn_euler_rk3_stage", U, U, None, ref, 1, 1e-4)
    torch.cuda.synchronize()
    assert np.array_equal(s, r)
    assert np.array_equal(_host(out), _host(ref))


def test_noalloc_stage_rejects_grid_above_limit(cn):
    lib = _abi()
    # 513 blocks of 32^3 cells = 32832 tiles of 8^3 > 32768
    U = cn.Grid.Cartesian((513, 1, 1), (32, 32, 32), ncomp=5, dtype=np.float32)
    sums = (C.c_double * 5)()
    rc = lib.cn_euler_rk3_stage_noalloc(U.handle, U.handle, None, U.handle, 1, 1e-3, GAMMA, sums, None)
    assert rc == CN_ERR_UNSUPPORTED
    assert "32768" in lib.cn_last_error_string().decode()
    rc = lib.cn_euler_rk3_stage_noalloc(U.handle, U.handle, None, U.handle, 1, 1e-3, GAMMA, None, None)
    assert rc == CN_ERR_INVALID_ARGUMENT  # sums_out is required
