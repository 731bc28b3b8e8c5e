"""K1 fused lab + FD stencils vs the reference loops / oracle (bit-exact: no
FMA contraction on either side)."""
import ctypes as C

import numpy as np
import pytest

from devgrid import make_grid
from golden_io import c1_small

pytestmark = pytest.mark.gpu


def _run(cn, op, g, outs):
    import torch
    getattr(cn.ops, op)(g, *outs)
    torch.cuda.synchronize()


def test_c1_small_matches_reference_loops(cn):
    c = c1_small()
    g = make_grid(cn, c["comp"], c["nb"], c["n"], begin=(0, 0, 0), end=(1, 1, 1))
    lap = cn.Grid.Cartesian(c["nb"], c["n"])
    grad = cn.Grid.Cartesian(c["nb"], c["n"], ncomp=3)
    _run(cn, "lap_grad", g, (lap, grad))
    assert np.array_equal(lap.download(0), c["lap"])
    for d in range(3):
        assert np.array_equal(grad.download(d), c["grad"][d])
    # separate operators give the same bits
    lap2 = cn.Grid.Cartesian(c["nb"], c["n"])
    grad2 = cn.Grid.Cartesian(c["nb"], c["n"], ncomp=3)
    _run(cn, "laplacian", g, (lap2,))
    _run(cn, "gradient", g, (grad2,))
    assert np.array_equal(lap2.download(0), c["lap"])
    for d in range(3):
        assert np.array_equal(grad2.download(d), c["grad"][d])


def _c1_field(O, nb, n, seed=1234):
    """u = sin(2 pi x) sin(2 pi y) cos(2 pi z) + U(-1e-3, 1e-3) at cell centres."""
    stride = O.block_stride(n, np.float64)
    nbk = int(np.prod(nb))
    comp = np.zeros(nbk * stride)
    h = [1.0 / (nb[d] * n[d]) for d in range(3)]
    rng = np.random.default_rng(seed)
    cells = int(np.prod(n))
    for b in range(nbk):
        bi = (b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1]))
        z, y, x = np.meshgrid(*[(np.arange(n[d]) + n[d] * bi[d] + 0.5) * h[d] for d in (2, 1, 0)],
                              indexing="ij")
        comp[b * stride:b * stride + cells] = (np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) *
                                               np.cos(2 * np.pi * z)).ravel()
    comp += rng.uniform(-1e-3, 1e-3, size=comp.size)
    return comp, h


@pytest.mark.parametrize("with_bc", [False, True])
def test_c1_full_size_vs_oracle(cn, oracle_lib, with_bc):
    """128^3 cells as 8^3 blocks of 16^3 (the C1 geometry), FP64."""
    O = oracle_lib
    nb, n = (8, 8, 8), (16, 16, 16)
    comp, h = _c1_field(O, nb, n)
    bcl = {}
    if with_bc:
        for b in range(512):
            bi = (b % 8, (b // 8) % 8, b // 64)
            lst = []
            if bi[1] == 0: lst.append((1, 0, O.BC_ABSORBING, 0))
            if bi[1] == 7: lst.append((1, 1, O.BC_SYMMETRY, -1))
            if bi[2] == 0: lst.append((2, 0, O.BC_DIRICHLET, 0.5))
            if bi[2] == 7: lst.append((2, 1, O.BC_DIRICHLET, -0.25))
            if lst: bcl[b] = lst
    g = make_grid(cn, comp, nb, n, bcl)
    lap = cn.Grid.Cartesian(nb, n)
    grad = cn.Grid.Cartesian(nb, n, ncomp=3)
    _run(cn, "lap_grad", g, (lap, grad))
    hh = g.getCellSize()
    want_lap = O.laplacian_f64(comp, nb, n, bcl, [1.0 / (x * x) for x in hh])
    want_grad = O.gradient_f64(comp, nb, n, bcl, [1.0 / x for x in hh])
    assert np.array_equal(lap.download(0), want_lap)
    for d in range(3):
        assert np.array_equal(grad.download(d), want_grad[d])
    # accuracy vs the exact Laplacian -12 pi^2 u (noise-free part), a sanity bound
    if not with_bc:
        cells = lap.blocks_view(lap.download(0))
        assert np.isfinite(cells).all()


def test_divergence_periodic_vs_numpy(cn, oracle_lib):
    O = oracle_lib
    nb, n = (3, 2, 2), (8, 4, 6)
    stride = O.block_stride(n, np.float64)
    nbk = int(np.prod(nb))
    rng = np.random.default_rng(5)
    g = cn.Grid.Cartesian(nb, n, ncomp=3)
    comps = [rng.standard_normal(nbk * stride) for _ in range(3)]
    for c in range(3):
        g.upload(comps[c], c)
    out = cn.Grid.Cartesian(nb, n)
    cn.ops.divergence(g, out)
    got = out.blocks_view(out.download(0))
    # global periodic arrays (z, y, x)
    def glob(a):
        v = a.reshape(nbk, stride)[:, : int(np.prod(n))].reshape(nb[2], nb[1], nb[0], n[2], n[1], n[0])
        return v.transpose(0, 3, 1, 4, 2, 5).reshape(nb[2] * n[2], nb[1] * n[1], nb[0] * n[0])
    v0, v1, v2 = (glob(a) for a in comps)
    ih = [1.0 / x for x in g.getCellSize()]
    t0 = (np.roll(v0, -1, 2) - np.roll(v0, 1, 2)) * ih[0]
    t1 = (np.roll(v1, -1, 1) - np.roll(v1, 1, 1)) * ih[1]
    t2 = (np.roll(v2, -1, 0) - np.roll(v2, 1, 0)) * ih[2]
    want = 0.5 * ((t0 + t1) + t2)
    gotg = got.reshape(nb[2], nb[1], nb[0], n[2], n[1], n[0]).transpose(0, 3, 1, 4, 2, 5).reshape(want.shape)
    assert np.array_equal(gotg, want)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_ddx_kernel_abi(cn, oracle_lib, dtype):
    """ISPC benchmark kernel ABI on a pitched 32^3 lab (BaseBenchmark.cpp:55-95)."""
    import torch
    N, g = 32, 1
    L = N + 2 * g
    xps = L + 6  # padded pitch like an aligned FieldLab row
    rng = np.random.default_rng(9)
    lab = rng.standard_normal((L, L, xps)).astype(dtype)
    dst = np.zeros((N, N, N), dtype=dtype)
    factor = dtype(1.0 / N)
    off = g + xps * (g + L * g)
    fn = oracle_lib.lib().or_ddx_f64 if dtype == np.float64 else oracle_lib.lib().or_ddx_f32
    CT = C.c_double if dtype == np.float64 else C.c_float
    fn.argtypes = [C.c_int] * 3 + [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, CT]
    fn(N, N, N, C.c_void_p(lab.ctypes.data + off * lab.itemsize), xps, xps * L,
       dst.ctypes.data_as(C.c_void_p), N, N * N, CT(factor))
    tlab = torch.from_numpy(lab).cuda()
    tdst = torch.zeros((N, N, N), dtype=tlab.dtype, device="cuda")
    lib = cn._lib.lib()
    f = lib.cn_ddx_f64 if dtype == np.float64 else lib.cn_ddx_f32
    f(N, N, N, C.c_void_p(tlab.data_ptr() + off * lab.itemsize), xps, xps * L,
      C.c_void_p(tdst.data_ptr()), N, N * N, factor)
    torch.cuda.synchronize()
    assert np.array_equal(tdst.cpu().numpy(), dst)


def _glob(a, nb, n, stride):
    """Block-ordered component -> global periodic array (z, y, x)."""
    nbk = int(np.prod(nb))
    v = a.reshape(nbk, stride)[:, : int(np.prod(n))].reshape(nb[2], nb[1], nb[0], n[2], n[1], n[0])
    return v.transpose(0, 3, 1, 4, 2, 5).reshape(nb[2] * n[2], nb[1] * n[1], nb[0] * n[0])


@pytest.mark.parametrize("n", [(5, 3, 7), (7, 6, 4), (6, 5, 3), (2, 9, 2)])
def test_lap_grad_odd_extents_vs_oracle(cn, oracle_lib, n):
    """Block extents with odd x (one cell per thread) and odd y / z (two cells
    per thread), periodic and with a BC chain, bit-exact vs the oracle."""
    O = oracle_lib
    nb = (3, 2, 2)
    stride = O.block_stride(n, np.float64)
    rng = np.random.default_rng(sum(n))
    comp = rng.standard_normal(int(np.prod(nb)) * stride)
    for bcl in ({}, {b: [(0, 0, O.BC_DIRICHLET, 0.25), (1, 1, O.BC_ABSORBING, 0), (2, 0, O.BC_SYMMETRY, -1)]
                     for b in range(int(np.prod(nb)))}):
        g = make_grid(cn, comp, nb, n, bcl)
        lap = cn.Grid.Cartesian(nb, n)
        grad = cn.Grid.Cartesian(nb, n, ncomp=3)
        _run(cn, "lap_grad", g, (lap, grad))
        hh = g.getCellSize()
        want_lap = O.laplacian_f64(comp, nb, n, bcl, [1.0 / (x * x) for x in hh])
        want_grad = O.gradient_f64(comp, nb, n, bcl, [1.0 / x for x in hh])
        assert np.array_equal(lap.download(0), want_lap)
        for d in range(3):
            assert np.array_equal(grad.download(d), want_grad[d])


@pytest.mark.parametrize("n", [(8, 4, 6), (5, 3, 7)])
def test_fp32_lap_grad_div_periodic_vs_numpy(cn, oracle_lib, n):
    """FP32 grids: the same operation order in float32 numpy (every operation
    rounded on its own, no contraction) gives the same bits."""
    O = oracle_lib
    nb = (3, 2, 2)
    stride = O.block_stride(n, np.float32)
    rng = np.random.default_rng(7)
    f32 = np.float32
    comps = [rng.standard_normal(int(np.prod(nb)) * stride).astype(f32) for _ in range(3)]
    g = cn.Grid.Cartesian(nb, n, ncomp=3, dtype=f32)
    for c in range(3):
        g.upload(comps[c], c)
    lap = cn.Grid.Cartesian(nb, n, dtype=f32)
    grad = cn.Grid.Cartesian(nb, n, ncomp=3, dtype=f32)
    div = cn.Grid.Cartesian(nb, n, dtype=f32)
    _run(cn, "lap_grad", g, (lap, grad))
    cn.ops.divergence(g, div)
    import torch
    torch.cuda.synchronize()
    hh = g.getCellSize()
    ih = [f32(1.0 / x) for x in hh]
    ih2 = [f32(1.0 / (x * x)) for x in hh]
    u = _glob(comps[0], nb, n, stride)
    xp, xm = np.roll(u, -1, 2), np.roll(u, 1, 2)
    yp, ym = np.roll(u, -1, 1), np.roll(u, 1, 1)
    zp, zm = np.roll(u, -1, 0), np.roll(u, 1, 0)
    c2 = f32(2) * u
    want_lap = (ih2[0] * ((xp - c2) + xm) + ih2[1] * ((yp - c2) + ym)) + ih2[2] * ((zp - c2) + zm)
    want_g = [f32(0.5) * ((xp - xm) * ih[0]), f32(0.5) * ((yp - ym) * ih[1]), f32(0.5) * ((zp - zm) * ih[2])]
    v0, v1, v2 = (_glob(a, nb, n, stride) for a in comps)
    t0 = (np.roll(v0, -1, 2) - np.roll(v0, 1, 2)) * ih[0]
    t1 = (np.roll(v1, -1, 1) - np.roll(v1, 1, 1)) * ih[1]
    t2 = (np.roll(v2, -1, 0) - np.roll(v2, 1, 0)) * ih[2]
    want_div = f32(0.5) * ((t0 + t1) + t2)
    assert np.array_equal(_glob(lap.download(0), nb, n, stride), want_lap)
    for d in range(3):
        assert np.array_equal(_glob(grad.download(d), nb, n, stride), want_g[d])
    assert np.array_equal(_glob(div.download(0), nb, n, stride), want_div)
