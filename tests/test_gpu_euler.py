"""K2 fused lab + WENO5-JS + Rusanov + divergence and the SSP-RK3 stages vs the
CPU oracle (same formulas; the device contracts multiply-adds and uses
refined approximate reciprocals, so results agree within the tolerances of
tests/numerics.py: 1e-13 relative in FP64), plus size-independent properties
at the full 512^3 size."""
import numpy as np
import pytest

from numerics import TOL_F32_RHS, TOL_F32_STATE, TOL_F64, assert_close

pytestmark = pytest.mark.gpu
GAMMA = 1.4


def _state(cn, nb, n, dtype, seed=7, bcs=True):
    U = cn.Grid.Cartesian(nb, n, ncomp=5, dtype=dtype)
    cn.workloads.euler_pulse(U, seed=seed)
    if bcs:
        cn.workloads.euler_bcs(U)
    return U


def _host(U):
    return np.stack([U.download(c) for c in range(5)])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("bcs", [True, False])
def test_rhs_matches_oracle(cn, oracle_lib, dtype, bcs):
    import torch
    nb, n = (2, 3, 2), (16, 8, 16)
    U = _state(cn, nb, n, dtype, bcs=bcs)
    R = cn.euler.like(U)
    cn.euler.rhs(U, R)
    torch.cuda.synchronize()
    host = _host(U)
    bcl = cn.workloads.euler_bclists(nb) if bcs else None
    want = oracle_lib.euler_stage(host, None, nb, n, bcl, 0, 0.0, GAMMA, U.getCellSize())
    got = _host(R)
    assert_close(got, want, TOL_F64 if dtype == np.float64 else TOL_F32_RHS,
                 f"rhs {np.dtype(dtype).name} bcs={bcs}")


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("stage", [1, 2, 3])
def test_stages_on_c2_blocks_match_oracle(cn, oracle_lib, dtype, stage):
    """2x2x2 blocks of 32^3 cells (the C2/C4 block size: 64 tiles per block,
    tiles on every block face and edge), C2 BCs, each SSP-RK3 stage."""
    import torch
    nb, n = (2, 2, 2), (32, 32, 32)
    U = _state(cn, nb, n, dtype, seed=21)
    Un = _state(cn, nb, n, dtype, seed=22)
    out = Un if stage == 3 else cn.euler.like(U)
    host, hn = _host(U), _host(Un)
    dt = 0.5 * cn.euler.cfl_dt(U, 0.3)
    cn.euler.rk3_stage(U, U, Un if stage > 1 else None, out, stage, dt)
    torch.cuda.synchronize()
    want = oracle_lib.euler_stage(host, hn if stage > 1 else None, nb, n, cn.workloads.euler_bclists(nb), stage,
                                  dt, GAMMA, U.getCellSize())
    got = _host(out)
    assert_close(got, want, TOL_F64 if dtype == np.float64 else TOL_F32_STATE,
                 f"stage {stage} {np.dtype(dtype).name} 32^3 blocks")


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_rk3_step_matches_oracle(cn, oracle_lib, dtype):
    import torch
    nb, n = (2, 2, 2), (16, 16, 16)
    U = _state(cn, nb, n, dtype)
    w1, w2 = cn.euler.like(U), cn.euler.like(U)
    host = _host(U)
    dt = cn.euler.cfl_dt(U, 0.3)
    sums = cn.euler.rk3_step(U, w1, w2, dt, want_sums=True)
    torch.cuda.synchronize()
    want = oracle_lib.euler_rk3_step(host, nb, n, cn.workloads.euler_bclists(nb), dt, GAMMA,
                                     U.getCellSize())
    got = _host(U)
    assert_close(got, want, TOL_F64 if dtype == np.float64 else TOL_F32_STATE,
                 f"rk3 step {np.dtype(dtype).name}")
    # FP64 conservation sums of U^{n+1}
    vol = np.prod(U.getCellSize())
    cells = int(np.prod(n))
    for c in range(5):
        ref = np.sum(U.blocks_view(got[c]).astype(np.float64)) * vol
        assert abs(sums[c] - ref) <= 1e-12 * max(1.0, abs(ref))


def test_fp32_vs_fp64_error(cn):
    """The FP32 form after a few RK3 steps stays within a stated error of FP64."""
    import torch
    nb, n = (2, 2, 2), (16, 16, 16)
    U64 = _state(cn, nb, n, np.float64)
    U32 = _state(cn, nb, n, np.float32)
    w = [cn.euler.like(U64), cn.euler.like(U64), cn.euler.like(U32), cn.euler.like(U32)]
    dt = cn.euler.cfl_dt(U64, 0.3)
    for _ in range(5):
        cn.euler.rk3_step(U64, w[0], w[1], dt)
        cn.euler.rk3_step(U32, w[2], w[3], dt)
    torch.cuda.synchronize()
    a, b = _host(U64), _host(U32).astype(np.float64)
    # errors relative to the magnitude of the state (rho ~ 1, E ~ 2.5): FP32
    # round-off accumulated over 5 RK3 steps
    scale = max(np.max(np.abs(a[0])), np.max(np.abs(a[4])))
    for c in range(5):
        l1 = np.mean(np.abs(a[c] - b[c])) / scale
        linf = np.max(np.abs(a[c] - b[c])) / scale
        print(f"var {c}: L1 {l1:.3e}  Linf {linf:.3e} (relative to max |state|)")
        assert linf < 1e-6 and l1 < 5e-7, (c, l1, linf)


def test_uniform_state_full_size_is_steady(cn):
    """512^3 cells (16^3 blocks of 32^3), C2 BCs: a uniform far-field state has
    an exactly zero RHS (every face sees the same six cells)."""
    import torch
    nb, n = (16, 16, 16), (32, 32, 32)
    U = cn.Grid.Cartesian(nb, n, ncomp=5)
    ff = cn.workloads.far_field()
    cells = 32 ** 3
    for c in range(5):
        U.tensor(c)[:, :cells].fill_(ff[c])
    cn.workloads.euler_bcs(U)
    R = cn.euler.like(U)
    cn.euler.rhs(U, R)
    torch.cuda.synchronize()
    for c in range(5):
        assert torch.count_nonzero(R.tensor(c)[:, :cells]).item() == 0
    del R, U
    torch.cuda.empty_cache()


def test_full_size_periodic_conservation_and_shift(cn):
    """512^3 periodic pulse: one RK3 step conserves every integral to round-off,
    and shifting the state by one block shifts the RHS bit for bit."""
    import torch
    nb, n = (16, 16, 16), (32, 32, 32)
    cells = 32 ** 3
    U = _state(cn, nb, n, np.float64, bcs=False)
    R = cn.euler.like(U)
    cn.euler.rhs(U, R)
    # shifted copy: block (bx,by,bz) -> (bx+1,by,bz)
    S = cn.euler.like(U)
    for c in range(5):
        src = U.tensor(c).view(16, 16, 16, -1)
        S.tensor(c).view(16, 16, 16, -1).copy_(torch.roll(src, shifts=1, dims=2))
    RS = cn.euler.like(U)
    cn.euler.rhs(S, RS)
    torch.cuda.synchronize()
    for c in range(5):
        want = torch.roll(R.tensor(c).view(16, 16, 16, -1), shifts=1, dims=2)[..., :cells]
        assert torch.equal(RS.tensor(c).view(16, 16, 16, -1)[..., :cells], want)
    del S, RS
    before = [U.tensor(c)[:, :cells].sum(dtype=torch.float64).item() for c in range(5)]
    dt = cn.euler.cfl_dt(U, 0.3)
    sums = cn.euler.rk3_step(U, R, cn.euler.like(U), dt, want_sums=True)
    vol = np.prod(U.getCellSize())
    for c in (0, 4):
        assert abs(sums[c] - before[c] * vol) <= 1e-12 * abs(before[c] * vol)
    del U, R
    torch.cuda.empty_cache()
