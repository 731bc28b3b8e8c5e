"""Multigrid operators vs the CPU oracle (bit-exact per kernel: same order, no
contraction), the coarsest FP64 CG within FP32 output round-off, and the
solver's convergence to a 1e-8 relative FP64 residual."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _end(nb, n):
    """Domain extent giving cubic cells (h = 1 / max cells)."""
    g = max(nb[d] * n[d] for d in range(3))
    return tuple(nb[d] * n[d] / g for d in range(3))


def _setup(cn, nb, n, seed=1):
    e = _end(nb, n)
    k = cn.Grid.Cartesian(nb, n, end=e, dtype=np.float32)
    cn.workloads.poisson_coefficient(k, seed=seed)
    f = cn.Grid.Cartesian(nb, n, end=e, dtype=np.float32)
    cn.workloads.poisson_rhs(f, seed=seed + 1)
    return k, f


# blocks of 8^3 (one tile per block) and of 32^3, the C5 block size (the
# 32x8x4 tile path, several tiles per block)
BLOCKS = [((2, 3, 2), (8, 8, 8)), ((2, 2, 2), (32, 32, 32))]


@pytest.mark.parametrize("nb,n", BLOCKS)
def test_jacobi_and_restriction_match_oracle(cn, oracle_lib, nb, n):
    import torch
    k, f = _setup(cn, nb, n)
    m = cn.mg.Multigrid(k, omega=0.8)
    p = cn.Grid.Cartesian(nb, n, end=_end(nb, n), dtype=np.float32)
    rng = np.random.default_rng(2)
    ph = np.zeros(p.comp_stride, dtype=np.float32)
    p.blocks_view(ph)[:] = rng.standard_normal(p.blocks_view(ph).shape)
    p.upload(ph)
    out = cn.Grid.Cartesian(nb, n, end=_end(nb, n), dtype=np.float32)
    m.jacobi(p, f, out)
    torch.cuda.synchronize()
    kh, fh = k.download(), f.download()
    ih2 = np.float32(1.0 / p.getCellSize()[0] ** 2)
    want = oracle_lib.mg_jacobi(ph, kh, fh, nb, n, 0.8, ih2)
    assert np.array_equal(p.blocks_view(out.download()), p.blocks_view(want))
    fc = m.level(1, "f")
    m.restrict_residual(p, f, fc)
    torch.cuda.synchronize()
    want = oracle_lib.mg_resid_restrict(ph, kh, fh, nb, n, ih2)
    assert np.array_equal(fc.blocks_view(fc.download()), fc.blocks_view(want))
    # coarse coefficients
    kc = m.level(1, "k")
    want = oracle_lib.mg_restrict_mean(kh, nb, n)
    assert np.array_equal(kc.blocks_view(kc.download()), kc.blocks_view(want))
    # prolongation of a random coarse correction
    ec = m.level(1, "p")
    eh = np.zeros(ec.comp_stride, dtype=np.float32)
    ec.blocks_view(eh)[:] = rng.standard_normal(ec.blocks_view(eh).shape)
    ec.upload(eh)
    m.prolong(ec, p)
    torch.cuda.synchronize()
    want = oracle_lib.mg_prolong(ph, eh, nb, n)
    assert np.array_equal(p.blocks_view(p.download()), p.blocks_view(want))


@pytest.mark.parametrize("nb,n", [((2, 2, 2), (8, 8, 8)), ((2, 2, 2), (32, 32, 32))])
def test_fp64_residual_matches_oracle(cn, oracle_lib, nb, n):
    import torch
    k, f = _setup(cn, nb, n)
    m = cn.mg.Multigrid(k)
    p64 = cn.Grid.Cartesian(nb, n, dtype=np.float64)
    rng = np.random.default_rng(3)
    ph = np.zeros(p64.comp_stride)
    p64.blocks_view(ph)[:] = rng.standard_normal(p64.blocks_view(ph).shape) * 1e-3
    p64.upload(ph)
    r32 = cn.Grid.Cartesian(nb, n, dtype=np.float32)
    rr, ff = m.residual(p64, f, r32)
    torch.cuda.synchronize()
    wr, wrr, wff = oracle_lib.mg_resid64(ph, k.download(), f.download(), nb, n, 1.0 / p64.getCellSize()[0] ** 2)
    assert np.array_equal(r32.blocks_view(r32.download()), r32.blocks_view(wr))
    assert abs(rr - wrr) <= 1e-12 * wrr and abs(ff - wff) <= 1e-12 * wff


def test_vcycle_and_coarsest_solve(cn, oracle_lib):
    """A 2-level cycle (coarsest = CG) against the oracle composition; the
    coarse FP64 CG differs from the oracle's only by summation order."""
    import torch
    nb, n = (4, 4, 4), (2, 2, 2)
    k, f = _setup(cn, nb, n)
    m = cn.mg.Multigrid(k, nu1=1, nu2=1, omega=0.8, max_levels=2)
    assert m.nlevels == 2 and m.coarsest_cells == 64
    e = cn.Grid.Cartesian(nb, n, dtype=np.float32)
    m.vcycle(f, e)
    torch.cuda.synchronize()
    kh, fh = k.download(), f.download()
    ih2 = np.float32(1.0 / e.getCellSize()[0] ** 2)
    p1 = oracle_lib.mg_jacobi(None, kh, fh, nb, n, 0.8, ih2)
    fc = oracle_lib.mg_resid_restrict(p1, kh, fh, nb, n, ih2)
    kc = oracle_lib.mg_restrict_mean(kh, nb, n)
    ec, _ = oracle_lib.mg_coarse_cg(fc, kc, nb, (1, 1, 1), 1.0 / (2 * e.getCellSize()[0]) ** 2)
    p2 = oracle_lib.mg_prolong(p1, ec, nb, n)
    want = oracle_lib.mg_jacobi(p2, kh, fh, nb, n, 0.8, ih2)
    got = e.download()
    scale = np.max(np.abs(want))
    assert np.max(np.abs(got - want)) <= 1e-5 * scale


@pytest.mark.parametrize("nb,n", [((4, 4, 4), (16, 16, 16)), ((8, 8, 8), (32, 32, 32))])
def test_solver_reaches_1e8(cn, nb, n):
    """64^3 and the full 256^3 problem: FP64 relative residual <= 1e-8."""
    import torch
    k, f = _setup(cn, nb, n)
    m = cn.mg.Multigrid(k, nu1=2, nu2=2, omega=0.8)
    p64 = cn.Grid.Cartesian(nb, n, dtype=np.float64)
    cycles, rel = m.solve(f, p64, rtol=1e-8, max_cycles=60)
    print(f"{nb}x{n}: {m.nlevels} levels, {cycles} cycles, relres {rel:.3e}")
    assert rel <= 1e-8 and cycles < 60
    rr, ff = m.residual(p64, f)
    assert np.sqrt(rr / ff) <= 1e-8
    del m, p64, k, f
    torch.cuda.empty_cache()


def test_manufactured_solution_second_order(cn):
    """k = 1, f = L_exact(u) for u = sin(2 pi x) sin(2 pi y) sin(2 pi z): the
    discrete solution converges to u at second order."""
    import torch
    errs = []
    for N in (32, 64):
        nb, n = (4, 4, 4), (N // 4,) * 3
        k = cn.Grid.Cartesian(nb, n, dtype=np.float32)
        k.tensor(0).fill_(1.0)
        f = cn.Grid.Cartesian(nb, n, dtype=np.float32)
        x = ((torch.arange(N, device="cuda", dtype=torch.float64) + 0.5) / N)
        s = torch.sin(2 * np.pi * x)
        u = s[:, None, None] * s[None, :, None] * s[None, None, :]
        cn.workloads._global_to_blocks(f, -12 * np.pi ** 2 * u, torch)
        m = cn.mg.Multigrid(k)
        p64 = cn.Grid.Cartesian(nb, n, dtype=np.float64)
        m.solve(f, p64, rtol=1e-10, max_cycles=60)
        got = torch.from_numpy(p64.download()).cuda()
        cells = int(np.prod(n))
        gv = got.view(p64.size(), -1)[:, :cells].reshape(4, 4, 4, n[2], n[1], n[0]).permute(0, 3, 1, 4, 2, 5).reshape(N, N, N)
        errs.append(float((gv - u).abs().max()))
    assert errs[1] < errs[0] / 3.0, errs


@pytest.mark.parametrize("nb,n", [((2, 2, 2), (16, 16, 16)), ((12, 12, 12), (2, 2, 2))])
def test_solve_matches_oracle_solve(cn, oracle_lib, nb, n):
    """The whole solve (V(2,2) cycles in FP64 defect correction) against the
    oracle's composition of the same operators: the same cycle count (the
    device's coarsest solve is exact up to round-off like the oracle's CG:
    the dense inverse on an 8-cell coarsest level, the FP64 CG on a
    1728-cell one) and the same solution up to the periodic constant, within
    1e-5 of its range."""
    import torch
    k, f = _setup(cn, nb, n)
    m = cn.mg.Multigrid(k, nu1=2, nu2=2, omega=0.8)
    p64 = cn.Grid.Cartesian(nb, n, dtype=np.float64)
    cycles, rel = m.solve(f, p64, rtol=1e-8, max_cycles=60)
    torch.cuda.synchronize()
    want, wc, wrel = oracle_lib.mg_solve(k.download(), f.download(), nb, n, k.getCellSize()[0], rtol=1e-8,
                                         max_cycles=60)
    assert abs(cycles - wc) <= 1 and rel <= 1e-8 and wrel <= 1e-8
    got = p64.blocks_view(p64.download())
    ref = p64.blocks_view(want)
    got, ref = got - got.mean(), ref - ref.mean()
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.ptp(ref)
