"""FaceContainer grids (Grid::Cartesian<T, Mesh, EntityType::Face, RANK>):
the structure of test/UnitTests/Grid/CartesianTest.cpp:46-103 (block ->
face direction -> component), the component map (block i, component c,
direction d) -> fields[i][d][c] of Block/FieldLabLoader.h:327-364, per-block
index ranges (Grid/BlockFieldAssembler.h:124-135), and the lab of every
direction and component through loadLab(field, lab, c, d), bit-exact against
the oracle (itself pinned to the reference's FieldLab on face fields)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
FACE = {0: 2, 1: 3, 2: 4}  # cn_entity of the face field of direction d


@pytest.mark.parametrize("ncomp", [1, 2])
def test_face_grid_structure_and_component_map(cn, ncomp):
    nb, n = (2, 3, 1), (4, 5, 6)
    g = cn.Grid.Cartesian(nb, n, entity="face", ncomp=ncomp)
    assert isinstance(g, cn.Grid.FaceCartesian)
    assert g.size() == 6 and tuple(g.getSize()) == nb and tuple(g.getBlockCells()) == n
    seen = set()
    nblk = 0
    for bf in g:  # FaceContainer of one block
        nblk += 1
        assert len(bf) == 3
        dirs = list(bf)
        assert len(dirs) == 3
        for d, f in enumerate(dirs):  # face field of direction d
            comps = [f] if ncomp == 1 else list(f)
            assert len(comps) == ncomp
            for c, fc in enumerate(comps):  # component of the face field
                assert fc.grid is g.faces[d] and fc.comp == c and fc.flat == bf.flat
                assert fc.grid.entity == "face_" + "xyz"[d]
                ptr = fc.grid.device_ptr(c) + bf.flat * fc.grid.block_stride * fc.grid.dtype.itemsize
                assert ptr % 32 == 0 and ptr not in seen
                seen.add(ptr)
                bi = fc.getState().block_index
                want = tuple(n[k] + (1 if k == d and bi[k] == nb[k] - 1 else 0) for k in range(3))
                assert tuple(fc.getIndexRange().getExtent()) == want
    assert nblk == 6
    for d in range(3):
        assert g.getBlockExtent(d) == tuple(n[k] + (k == d) for k in range(3))
        for c in range(ncomp):
            f = g.getIndexFunctor(c, d)((1, 2, 0))
            assert f.grid is g.faces[d] and f.comp == c and f.flat == g.flat_index((1, 2, 0))
            f2 = g.field((1, 2, 0), c, d)
            assert f2.grid is f.grid and f2.comp == c and f2.flat == f.flat
    with pytest.raises(IndexError):
        g[0][3]
    g.close()


def test_face_container_labs_vs_oracle(cn, oracle_lib):
    import torch
    O = oracle_lib
    rng = np.random.default_rng(77)
    for trial in range(6):
        nb = [int(v) for v in rng.integers(1, 4, size=3)]
        cells = [int(v) for v in rng.integers(2, 6, size=3)]
        ncomp = int(rng.integers(1, 3))
        lo = [int(rng.integers(0, cells[d] + 1)) for d in range(3)]
        hi = [int(rng.integers(1, cells[d] + 1)) for d in range(3)]
        tens = bool(rng.integers(0, 2))
        g = cn.Grid.Cartesian(nb, cells, entity="face", ncomp=ncomp)
        nblocks = g.size()
        host, bcls = {}, {}
        for d in range(3):
            code = FACE[d]
            stride = O.entity_stride(cells, code, np.float64)
            assert g.faces[d].block_stride == stride
            for c in range(ncomp):
                comp = rng.standard_normal(nblocks * stride) * 10
                g.upload(comp, c, d)
                bcl = {b: [(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 4)),
                            float(rng.choice([-1, 0.5, 2]))) for _ in range(int(rng.integers(0, 3)))]
                       for b in range(nblocks)}
                for b, lst in bcl.items():
                    for (dd, s, k, v) in lst:
                        C_ = {0: cn.BC.Base, 1: cn.BC.Dirichlet, 2: cn.BC.Absorbing, 3: cn.BC.Symmetry}[k]
                        g.field(b, c, d).getBC().push_back(C_(dd, s) if k in (0, 2) else C_(dd, s, v))
                host[d, c], bcls[d, c] = comp, bcl
        stencil = cn.Core.Stencil([-v for v in lo], [v + 1 for v in hi], tens)
        for d in range(3):
            code = FACE[d]
            n = g.getBlockExtent(d)
            stride = g.faces[d].block_stride
            lab = cn.Block.FieldLab()
            lab.allocate(stencil, cn.Core.IndexRange(n))
            for c in range(ncomp):
                for b in range(nblocks):
                    bf = g[b]
                    g.loadLab(bf, lab, c, d)
                    torch.cuda.synchronize()
                    want, wdef = O.lab_fill(host[d, c], nb, n, lo, hi, tens, bcls[d, c], b, stride=stride,
                                            entity=code)
                    got = lab.data.cpu().numpy()
                    act = [ext + lo[k] + hi[k] for k, ext in enumerate(g.faces[d].block_extent(b))]
                    assert list(got.shape) == act[::-1]
                    assert tuple(lab.getActiveRange().getExtent()) == tuple(g.faces[d].block_extent(b))
                    # the active lab range of this block: the oracle's lab has
                    # the strides of the largest lab, as the device's has
                    want = want[: act[2], : act[1], : act[0]]
                    wdef = wdef[: act[2], : act[1], : act[0]].astype(bool)
                    assert wdef.any()
                    assert np.array_equal(got[wdef].view(np.uint8), want[wdef].view(np.uint8)), (trial, d, c, b)
        g.close()
