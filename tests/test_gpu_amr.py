"""Two-level AMR layouts: interface ghost fill (bit-exact) and the fused
Euler stage (within the FP64 tolerance of tests/numerics.py) vs the CPU
oracle, a steady uniform state at the full size, schedule independence, and
CUDA-graph replay of the RK3 step."""
import numpy as np
import pytest

from numerics import TOL_F32_RHS, TOL_F32_STATE, TOL_F64, assert_close

pytestmark = pytest.mark.gpu
GAMMA = 1.4


def _small(cn, seed=3):
    l, c, o, F = cn.workloads.amr_small_layout(seed)
    U = cn.amr.AmrGrid(l, c, o, F)
    return U, l, c, o, F


def test_amr_lab_fill_matches_oracle(cn, oracle_lib):
    import torch
    U, l, c, o, F = _small(cn)
    blk, tot = oracle_lib.amr_blocks(l, c, o, F)
    assert tot == U.total_cells
    rng = np.random.default_rng(4)
    comp = rng.standard_normal(tot)
    U.upload(comp, 0)
    kinds = set()
    for b in range(U.nblocks):
        got = U.lab(0, 3, b, fill=np.nan).cpu().numpy()
        want, w = oracle_lib.amr_lab(comp, blk, F, b, 3)
        assert np.array_equal(got[w], want[w]), b
        kinds.add((int(l[b]), int(c[b])))
    assert len(kinds) >= 3


@pytest.mark.parametrize("stage", [0, 1, 2, 3])
def test_amr_stage_matches_oracle(cn, oracle_lib, stage):
    import torch
    U, l, c, o, F = _small(cn)
    cn.workloads.euler_pulse_amr(U, seed=7)
    Un = U.like()
    cn.workloads.euler_pulse_amr(Un, seed=8)
    out = U.like()
    host = np.stack([U.download(k) for k in range(5)])
    hn = np.stack([Un.download(k) for k in range(5)])
    if stage == 3:
        out = Un  # stage 3 writes over U^n
    cn.amr.rk3_stage(U, Un if stage > 1 else None, out, stage, 2e-4, GAMMA)
    torch.cuda.synchronize()
    blk, _ = oracle_lib.amr_blocks(l, c, o, F)
    want = oracle_lib.amr_stage(host, hn if stage > 1 else None, blk, F, stage, 2e-4, GAMMA)
    got = np.stack([out.download(k) for k in range(5)])
    assert_close(got, want, TOL_F64, f"amr stage {stage}")


@pytest.mark.parametrize("stage", [0, 1, 3])
def test_amr_stage_fp32_matches_fp64_oracle(cn, oracle_lib, stage):
    """The FP32 AMR stage (interface ghosts and WENO5 in FP32) against the
    FP64 oracle on the same FP32-rounded inputs: the FP32 tolerances of
    tests/numerics.py (right-hand side, and stage updates)."""
    import torch
    l, c, o, F = cn.workloads.amr_small_layout(3)
    U = cn.amr.AmrGrid(l, c, o, F, dtype=np.float32)
    cn.workloads.euler_pulse_amr(U, seed=7)
    Un = U.like()
    cn.workloads.euler_pulse_amr(Un, seed=8)
    out = U.like()
    host = np.stack([U.download(k) for k in range(5)]).astype(np.float64)
    hn = np.stack([Un.download(k) for k in range(5)]).astype(np.float64)
    if stage == 3:
        out = Un
    cn.amr.rk3_stage(U, Un if stage > 1 else None, out, stage, 2e-4, GAMMA)
    torch.cuda.synchronize()
    blk, _ = oracle_lib.amr_blocks(l, c, o, F)
    want = oracle_lib.amr_stage(host, hn if stage > 1 else None, blk, F, stage, 2e-4, GAMMA)
    got = np.stack([out.download(k) for k in range(5)]).astype(np.float64)
    assert_close(got, want, TOL_F32_RHS if stage == 0 else TOL_F32_STATE, f"amr float32 stage {stage}")


def test_amr_schedules_and_graph_are_bitwise_identical(cn):
    import torch
    U, *_ = _small(cn)
    cn.workloads.euler_pulse_amr(U, seed=9)
    w1, w2 = U.like(), U.like()
    start = [U.tensor(k).clone() for k in range(5)]
    results = []
    shapes = [(1, 1, 1), (2, 1, 1), (4, 1, 1), (1, 2, 1), (1, 1, 2), (2, 2, 1), (2, 2, 2), (4, 4, 4)]
    for shape in shapes:
        for order in range(3):
            for ctas in (0, 148 * 3):
                for k in range(5):
                    U.tensor(k).copy_(start[k])
                for g in (U, w1, w2):
                    g.set_schedule(order, ctas, shape=shape)
                    assert g.work_shape() == shape
                    assert g.schedule() == (order, ctas, shape[0] * shape[1] * shape[2])
                cn.amr.rk3_step(U, w1, w2, 1e-4, GAMMA)
                torch.cuda.synchronize()
                results.append(torch.cat([U.tensor(k).clone() for k in range(5)]))
    for g in (U, w1, w2):
        g.set_schedule(1, 0, 2)  # the unit form: shape (2, 1, 1)
        assert g.work_shape() == (2, 1, 1)
        g.set_schedule(1, 0, 1)
    for r in results[1:]:
        assert torch.equal(r, results[0])
    # graph replay of the step
    s = torch.cuda.Stream()
    for k in range(5):
        U.tensor(k).copy_(start[k])
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        cn.amr.rk3_step(U, w1, w2, 1e-4, GAMMA, stream=s)  # eager once
    s.synchronize()
    for k in range(5):
        U.tensor(k).copy_(start[k])
    torch.cuda.synchronize()
    g = cn.amr.Graph.capture(lambda: cn.amr.rk3_step(U, w1, w2, 1e-4, GAMMA, stream=s), s)
    g.launch(s)
    s.synchronize()
    got = torch.cat([U.tensor(k).clone() for k in range(5)])
    assert torch.equal(got, results[0])


@pytest.mark.parametrize("stage", [0, 2])
def test_amr_rectangular_box_matches_oracle(cn, oracle_lib, stage):
    """A small layout of the batched-AMR recipe (40 blocks of all three sizes
    on both levels, periodic box of 160 x 128 x 64 level-1 cells): labs of
    every block bit for bit and the stage within the FP64 tolerance."""
    import torch
    l, c, o, F = cn.workloads.amr_layout(1, nblocks=40)
    assert tuple(F) == (160, 128, 64)
    U = cn.amr.AmrGrid(l, c, o, F)
    blk, tot = oracle_lib.amr_blocks(l, c, o, F)
    assert tot == U.total_cells
    cn.workloads.euler_pulse_amr(U, seed=11)
    Un = U.like()
    cn.workloads.euler_pulse_amr(Un, seed=12)
    host = np.stack([U.download(k) for k in range(5)])
    hn = np.stack([Un.download(k) for k in range(5)])
    for b in range(U.nblocks):
        got = U.lab(0, 3, b, fill=np.nan).cpu().numpy()
        want, w = oracle_lib.amr_lab(host[0], blk, F, b, 3)
        assert np.array_equal(got[w], want[w]), b
    out = U.like()
    cn.amr.rk3_stage(U, Un if stage > 1 else None, out, stage, 1e-4, GAMMA)
    torch.cuda.synchronize()
    want = oracle_lib.amr_stage(host, hn if stage > 1 else None, blk, F, stage, 1e-4, GAMMA)
    got = np.stack([out.download(k) for k in range(5)])
    assert_close(got, want, TOL_F64, f"amr box stage {stage}")


def test_amr_full_layout_uniform_state_is_steady(cn):
    """The batched layout (2048 blocks of 8^3/16^3/32^3 cells, about 13.5 M
    cells): a uniform state with exactly representable values has an exactly
    zero RHS (ghosts interpolate exactly)."""
    import torch
    l, c, o, F = cn.workloads.amr_layout()
    U = cn.amr.AmrGrid(l, c, o, F)
    vals = (1.0, 0.5, -0.25, 0.0, 2.5)
    for k in range(5):
        U.tensor(k).fill_(vals[k])
    R = U.like()
    cn.amr.rk3_stage(U, None, R, 0, 0.0, GAMMA)
    torch.cuda.synchronize()
    for k in range(5):
        assert torch.count_nonzero(R.tensor(k)).item() == 0
