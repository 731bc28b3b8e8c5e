"""K0 device lab fill vs the reference FieldLab (bit-exact), through the C ABI."""
import numpy as np
import pytest

import labchecks as LC
from devgrid import lab_fill_all, make_grid
from golden_io import lab_cases

pytestmark = pytest.mark.gpu
CASES = lab_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_lab_fill_matches_reference_golden(cn, case):
    g = make_grid(cn, case["comp"], case["nb"], case["n"], case["bcs"])
    labs, written = lab_fill_all(cn, g, case["lo"], case["hi"], case["tensorial"])
    for i, b in enumerate(case["blocks"]):
        LC.compare_defined(labs[b], written[b], case["labs"][i], case["defined"][i])


def test_lab_fill_randomised_vs_oracle(cn, oracle_lib):
    O = oracle_lib
    rng = np.random.default_rng(11)
    for trial in range(150):
        dt = [np.float64, np.float32, np.int32][trial % 3]
        nb = rng.integers(1, 4, size=3)
        n = rng.integers(1, 7, size=3)
        lo = [int(rng.integers(0, n[d] + 1)) for d in range(3)]
        hi = [int(rng.integers(0, n[d] + 1)) for d in range(3)]
        tens = bool(rng.integers(0, 2))
        nblocks = int(np.prod(nb))
        stride = O.block_stride(n, dt)
        if dt == np.int32:
            comp = rng.integers(-1000, 1000, size=nblocks * stride).astype(dt)
        else:
            comp = (rng.standard_normal(nblocks * stride) * 100).astype(dt)
        bcl = {b: [(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 4)),
                    float(rng.choice([-3, -1, 0.5, 1, 2]))) for _ in range(int(rng.integers(0, 6)))]
               for b in range(nblocks)}
        g = make_grid(cn, comp, nb, n, bcl)
        labs, written = lab_fill_all(cn, g, lo, hi, tens)
        for b in range(nblocks):
            want, wdef = O.lab_fill(comp, nb, n, lo, hi, tens, bcl, b)
            LC.compare_defined(labs[b], written[b], want, wdef)
        g.close()


def test_lab_fill_without_bc_keeps_skips(cn, oracle_lib):
    """loadData(..., apply_bc=false): neighbours are still skipped where a BC
    exists (Block/FieldLab.h:206-216) but no BC is applied."""
    nb, n = (2, 2, 2), (4, 4, 4)
    comp = np.arange(8 * 64, dtype=np.float64)
    bcl = {b: [(1, 0, 1, 5.0)] for b in range(8)}
    g = make_grid(cn, comp, nb, n, bcl)
    labs, written = lab_fill_all(cn, g, (1, 1, 1), (1, 1, 1), False, apply_bc=False)
    # the y-low face is skipped and not written
    assert not written[0][1:5, 0, 1:5].any()
    assert written[0][1:5, 5, 1:5].all()
    g.close()


def test_c1_shaped_grid_vs_oracle(cn, oracle_lib):
    """Full C1 geometry: 8^3 blocks of 16^3, stencil (-1,2), FP64."""
    O = oracle_lib
    nb, n = (8, 8, 8), (16, 16, 16)
    rng = np.random.default_rng(3)
    stride = O.block_stride(n, np.float64)
    comp = rng.standard_normal(512 * stride)
    g = make_grid(cn, comp, nb, n)
    labs, written = lab_fill_all(cn, g, (1, 1, 1), (1, 1, 1), False)
    for b in list(range(0, 512, 37)) + [511]:
        want, wdef = O.lab_fill(comp, nb, n, (1, 1, 1), (1, 1, 1), False, {}, b)
        LC.compare_defined(labs[b], written[b], want, wdef)
    g.close()


def test_fieldlab_api_interface(cn):
    """FieldLabTest.cpp:223-291 through the Python mirror of Block::FieldLab."""
    n = (16, 16, 1)
    g = cn.Grid.Cartesian((1, 1, 1), (16, 16, 4), dtype=np.int32)
    host = np.zeros(g.comp_stride, dtype=np.int32)
    host[: 16 * 16 * 4] = np.arange(16 * 16 * 4)
    g.upload(host)
    lab = cn.Block.FieldLab()
    fp = lab.getMemoryFootprint()
    assert fp.allocated == 0 and fp.used == 0
    with pytest.raises(RuntimeError, match="^FieldLab: no field loaded$"):
        lab.getActiveField()
    with pytest.raises(RuntimeError, match="^FieldLab: can not load lab data when not allocated first$"):
        lab.loadData(0, g)
    s = cn.Core.Stencil(-3, 4)
    lab.allocate(s, g[0].getIndexRange())
    g.loadLab(g[0], lab)
    assert lab[(0, 0, 0)] == host[0]
    assert lab.getActiveStencil() == s
    assert lab.getActiveRange().getExtent() == (16, 16, 4)
    assert lab.getActiveField().flat == 0
    lr = lab.getActiveLabRange()
    assert lr.getBegin() == (-3, -3, -3)
    assert lr.getEnd() == (16 + 3, 16 + 3, 4 + 3)
    assert lab.getMemoryFootprint().used == lr.size() * 4
    g.close()


def test_grid_bc_vector_api(cn):
    """Field::getBC() vector semantics (Block/Field.h:437-442)."""
    g = cn.Grid.Cartesian((2, 2, 2), (4, 4, 4))
    f = g[(1, 0, 0)]
    f.getBC().push_back(cn.BC.Dirichlet(0, 1, 3.0))
    f.getBC().push_back(cn.BC.Absorbing(1, 0))
    assert len(f.getBC()) == 2
    assert [b.name() for b in f.getBC()] == ["Dirichlet", "Zeroth-Order Absorbing"]
    f.getBC().clear()
    assert len(g[(1, 0, 0)].getBC()) == 0
    other = cn.Grid.Cartesian((2, 2, 1), (4, 4, 4))
    with pytest.raises(RuntimeError, match="^Cartesian: Can not assign two grids of unequal size.$"):
        other.copy_from(g)
    with pytest.raises(RuntimeError, match="ghost width"):
        lab = cn.Block.FieldLab()
        lab.allocate(cn.Core.Stencil(-5, 2), g[0].getIndexRange())
        g.loadLab(g[0], lab)
    g.close()
    other.close()


def test_load_labs_c2_geometry_vs_oracle(cn, oracle_lib):
    """ops.load_labs (all blocks in one launch) on the lab workload's geometry,
    reduced to 4x4x2 blocks of 32^3: the Euler pulse state, C2 BCs (y
    absorbing, z Dirichlet per component), stencil (-3,4) non-tensorial; every
    block's defined lab cells bit-exact against the oracle."""
    import torch
    O = oracle_lib
    nb, n = (4, 4, 2), (32, 32, 32)
    U = cn.Grid.Cartesian(nb, n, ncomp=5)
    cn.workloads.euler_pulse(U)
    cn.workloads.euler_bcs(U)
    bcl = cn.workloads.euler_bclists(nb)
    st = cn.Core.Stencil(-3, 4, False)
    for c in (0, 4):
        labs = cn.ops.load_labs(U, st, comp=c)
        torch.cuda.synchronize()
        host = labs.cpu().numpy()
        comp = U.download(c)
        for b in range(int(np.prod(nb))):
            want, wdef = O.lab_fill(comp, nb, n, (3, 3, 3), (3, 3, 3), False, bcl[c], b)
            assert np.array_equal(host[b][wdef], want[wdef]), (c, b)
    # a block range: blocks 5..9 land in out[0..4]
    part = cn.ops.load_labs(U, st, comp=2, block_begin=5, count=5)
    full = cn.ops.load_labs(U, st, comp=2)
    torch.cuda.synchronize()
    comp = U.download(2)
    for i in range(5):
        _, wdef = O.lab_fill(comp, nb, n, (3, 3, 3), (3, 3, 3), False, bcl[2], 5 + i)
        assert torch.equal(part[i][torch.from_numpy(wdef).cuda()], full[5 + i][torch.from_numpy(wdef).cuda()])
    U.close()


def test_lab_fill_long_rows_vs_oracle(cn, oracle_lib):
    """Blocks whose lab slabs hold more ghost rows than the kernel resolves in
    one round (2 x 200 x 6 cells: slabs of 208 and 204 ghost rows against a
    table of 96), with BCs and skips on every face, non-tensorial and
    tensorial: bit-exact against the oracle."""
    O = oracle_lib
    rng = np.random.default_rng(21)
    nb, n = (2, 2, 2), (2, 200, 6)
    nblocks = 8
    stride = O.block_stride(n, np.float64)
    comp = rng.standard_normal(nblocks * stride)
    bcl = {b: [(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 4)),
                float(rng.choice([-1, 0.5, 2]))) for _ in range(3)] for b in range(nblocks) if b % 2}
    for tens in (False, True):
        g = make_grid(cn, comp, nb, n, bcl)
        labs, written = lab_fill_all(cn, g, (1, 1, 1), (1, 1, 1), tens)
        for b in range(nblocks):
            want, wdef = O.lab_fill(comp, nb, n, (1, 1, 1), (1, 1, 1), tens, bcl, b)
            LC.compare_defined(labs[b], written[b], want, wdef)
        g.close()


def test_lab_fill_thinner_slabs_vs_oracle(cn, oracle_lib):
    """Blocks of 4 x 40 x 6 cells with two ghost planes along z: a slab of the
    whole lab (10 planes) holds 172 ghost rows, more than the one-pass
    kernel's table, so the host takes slabs of 8 planes (92 and 80 rows) and
    keeps that kernel; BCs on some faces, bit-exact against the oracle."""
    O = oracle_lib
    rng = np.random.default_rng(31)
    nb, n, lo, hi = (2, 2, 2), (4, 40, 6), (1, 1, 2), (1, 1, 2)
    nblocks = 8
    for dt in (np.float64, np.float32):
        stride = O.block_stride(n, dt)
        comp = (rng.standard_normal(nblocks * stride) * 10).astype(dt)
        bcl = {b: [(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 4)),
                    float(rng.choice([-1, 0.5, 2]))) for _ in range(2)] for b in range(nblocks) if b % 3 == 0}
        g = make_grid(cn, comp, nb, n, bcl)
        labs, written = lab_fill_all(cn, g, lo, hi, False)
        for b in range(nblocks):
            want, wdef = O.lab_fill(comp, nb, n, lo, hi, False, bcl, b)
            LC.compare_defined(labs[b], written[b], want, wdef)
        g.close()
