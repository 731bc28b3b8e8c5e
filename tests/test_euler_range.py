"""WENO5-JS weights at the magnitudes of dimensional (SI) data.

The weight products t_i t_j of a jump J grow like 20 J^8, which leaves the
FP32 range above J ~ 4e4: a pressure jump of one bar in pascals.  FP32 forms
them from the smoothness sums rescaled by an exact power of two (largest and
middle exponent), so the FP32 Euler RHS stays finite and tracks FP64 at any
pressure scale.  CPU tests check the oracle; GPU tests check the device
against the oracle on the same data, within the tolerances of
tests/numerics.py."""
import numpy as np
import pytest

import oracle as O
from numerics import TOL_F32_RHS, TOL_F32_STATE, TOL_F64, assert_close

GAMMA = 1.4
PRESSURES = [1e5, 1e9, 1e12]  # Pa: one bar, 10 kbar, 10 Mbar
NB, N = (2, 2, 1), (16, 8, 16)


def _to_blocks(glob, nb, n, stride):
    """Global (z, y, x) array -> component array in grid layout (blocks x
    fastest, cells x fastest inside a block, blocks padded to `stride`)."""
    nbx, nby, nbz = nb
    nx, ny, nz = n
    a = glob.reshape(nbz, nz, nby, ny, nbx, nx).transpose(0, 2, 4, 1, 3, 5).reshape(nbx * nby * nbz, nx * ny * nz)
    out = np.zeros((a.shape[0], stride), glob.dtype)
    out[:, : a.shape[1]] = a
    return out.ravel()


def si_state(P, dtype, nb=NB, n=N, seed=3):
    """Two-state shock-tube data in SI units: density 1.2 / 0.15 kg/m^3 with a
    smooth bump, pressure P / 0.1 P across two planes, random velocities up to
    a tenth of the sound speed.  Returns (5, nblocks * stride) conservative
    components."""
    rng = np.random.default_rng(seed)
    cells = [nb[d] * n[d] for d in range(3)]
    z, y, x = np.meshgrid(*[(np.arange(cells[d]) + 0.5) / cells[d] for d in (2, 1, 0)], indexing="ij")
    left = (x < 0.5) ^ (y < 0.3)
    rho = np.where(left, 1.2, 0.15) * (1 + 0.3 * np.exp(-((x - 0.3) ** 2 + (z - 0.6) ** 2) / 0.02))
    p = np.where(left, 1.0, 0.1) * P
    c = np.sqrt(GAMMA * P / 1.2)
    vel = [0.1 * c * (rng.random(rho.shape) * 2 - 1) for _ in range(3)]
    E = p / (GAMMA - 1) + 0.5 * rho * (vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)
    stride = O.block_stride(n, np.dtype(dtype))
    comps = [rho, rho * vel[0], rho * vel[1], rho * vel[2], E]
    return np.stack([_to_blocks(q.astype(dtype), nb, n, stride) for q in comps])


def _cells(a, n, dtype):
    st = O.block_stride(n, np.dtype(dtype))
    return a.reshape(5, -1, st)[:, :, : int(np.prod(n))]


H = tuple(1.0 / (NB[d] * N[d]) for d in range(3))


@pytest.mark.parametrize("P", PRESSURES)
def test_oracle_fp32_rhs_finite_and_tracks_fp64(P):
    r64 = _cells(O.euler_stage(si_state(P, np.float64), None, NB, N, None, 0, 0.0, GAMMA, H), N, np.float64)
    r32 = _cells(O.euler_stage(si_state(P, np.float32), None, NB, N, None, 0, 0.0, GAMMA, H), N, np.float32)
    assert np.isfinite(r64).all() and np.isfinite(r32).all()
    for c in range(5):
        # FP32 inputs are the FP64 data rounded once; the RHS differs by
        # round-off (observed below 1e-6 of max |R_c|)
        rel = np.max(np.abs(r32[c].astype(np.float64) - r64[c])) / np.max(np.abs(r64[c]))
        assert rel < 4e-6, (P, c, rel)


def test_oracle_fp32_rk3_step_si_units():
    """Three SSP-RK3 steps of the shock-tube data at one bar stay finite and
    within FP32 round-off of FP64 (relative to the state's magnitude)."""
    U64, U32 = si_state(1e5, np.float64), si_state(1e5, np.float32)
    c = np.sqrt(GAMMA * 1e5 / 0.15)
    dt = 0.3 * min(H) / (1.1 * c)
    for _ in range(3):
        U64 = O.euler_rk3_step(U64, NB, N, None, dt, GAMMA, H)
        U32 = O.euler_rk3_step(U32, NB, N, None, dt, GAMMA, H)
    a, b = _cells(U64, N, np.float64), _cells(U32, N, np.float32).astype(np.float64)
    assert np.isfinite(b).all()
    for k in range(5):
        rel = np.max(np.abs(a[k] - b[k])) / np.max(np.abs(a[k]))
        assert rel < 1e-5, (k, rel)


def _device_state(cn, host, dtype):
    U = cn.Grid.Cartesian(NB, N, ncomp=5, dtype=dtype)
    for c in range(5):
        U.upload(host[c], c)
    return U


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("P", PRESSURES)
def test_device_rhs_si_units_matches_oracle(cn, oracle_lib, P, dtype):
    import torch
    host = si_state(P, dtype)
    U = _device_state(cn, host, dtype)
    R = cn.euler.like(U)
    cn.euler.rhs(U, R)
    torch.cuda.synchronize()
    want = oracle_lib.euler_stage(host, None, NB, N, None, 0, 0.0, GAMMA, U.getCellSize())
    got = np.stack([R.download(c) for c in range(5)])
    assert_close(_cells(got, N, dtype), _cells(want, N, dtype),
                 TOL_F64 if dtype == np.float64 else TOL_F32_RHS, f"SI rhs P={P:g} {np.dtype(dtype).name}")


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_device_rk3_step_si_units_matches_oracle(cn, oracle_lib, dtype):
    import torch
    host = si_state(1e5, dtype)
    U = _device_state(cn, host, dtype)
    w1, w2 = cn.euler.like(U), cn.euler.like(U)
    dt = cn.euler.cfl_dt(U, 0.3)
    cn.euler.rk3_step(U, w1, w2, dt)
    torch.cuda.synchronize()
    want = oracle_lib.euler_rk3_step(host, NB, N, None, dt, GAMMA, U.getCellSize())
    got = np.stack([U.download(c) for c in range(5)])
    assert_close(_cells(got, N, dtype), _cells(want, N, dtype),
                 TOL_F64 if dtype == np.float64 else TOL_F32_STATE, f"SI rk3 step {np.dtype(dtype).name}")
