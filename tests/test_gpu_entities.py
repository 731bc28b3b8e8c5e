"""Node and face fields (Grid::Cartesian<T, Mesh, EntityType::Node|Face>):
the device lab fill against the C oracle, which is pinned to the reference's
FieldLab on the same fields (tests/test_oracle.py); bit for bit, defined
cells included.  Only the last block along a grown dimension holds cells + 1
entities (Grid/BlockFieldAssembler.h:124-135)."""
import numpy as np
import pytest

import labchecks as LC
from devgrid import lab_fill_all, make_grid

pytestmark = pytest.mark.gpu
ENTITIES = {"node": 1, "face_x": 2, "face_y": 3, "face_z": 4}


@pytest.mark.parametrize("entity", list(ENTITIES))
def test_entity_lab_fill_vs_oracle(cn, oracle_lib, entity):
    O = oracle_lib
    code = ENTITIES[entity]
    rng = np.random.default_rng(31 + code)
    for trial in range(30):
        nb = [int(v) for v in rng.integers(1, 4, size=3)]
        cells = [int(v) for v in rng.integers(2, 7, size=3)]
        n = [c + g for c, g in zip(cells, O.ENTITY_GROW[code])]
        lo = [int(rng.integers(0, cells[d] + 1)) for d in range(3)]
        hi = [int(rng.integers(0, cells[d] + 1)) for d in range(3)]
        tens = bool(rng.integers(0, 2))
        nblocks = int(np.prod(nb))
        stride = O.entity_stride(cells, code, np.float64)
        comp = rng.standard_normal(nblocks * stride) * 100
        bcl = {b: [(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 4)),
                    float(rng.choice([-3, -1, 0.5, 1, 2]))) for _ in range(int(rng.integers(0, 5)))]
               for b in range(nblocks)}
        g = make_grid(cn, comp, nb, cells, bcl, entity=entity)
        assert g.getBlockExtent() == tuple(n) and g.block_stride == stride
        labs, written = lab_fill_all(cn, g, lo, hi, tens)
        for b in range(nblocks):
            want, wdef = O.lab_fill(comp, nb, n, lo, hi, tens, bcl, b, stride=stride, entity=code)
            LC.compare_defined(labs[b], written[b], want, wdef)
        g.close()


def test_node_grid_periodic_identities(cn):
    """FieldLabTest.cpp:56-100 (there 2-D) on a one-block node grid: every
    ghost equals the value one extent (cells + 1) away."""
    import torch
    cells = (8, 8, 8)
    n = tuple(c + 1 for c in cells)
    g = cn.Grid.Cartesian((1, 1, 1), cells, entity="node")
    comp = np.zeros(g.comp_stride)
    comp[: int(np.prod(n))] = np.arange(int(np.prod(n)), dtype=np.float64)
    g.upload(comp)
    for tens in (False, True):
        labs, written = lab_fill_all(cn, g, (2, 2, 2), (2, 2, 2), tens)
        torch.cuda.synchronize()
        f = comp[: int(np.prod(n))].reshape(n[2], n[1], n[0])
        lab = LC.Lab(labs[0], n, (2, 2, 2), (2, 2, 2))
        w = LC.Lab(written[0], n, (2, 2, 2), (2, 2, 2))
        for z in range(-2, n[2] + 2):
            for y in range(-2, n[1] + 2):
                for x in range(-2, n[0] + 2):
                    if w[(x, y, z)]:
                        assert lab[(x, y, z)] == f[z % n[2], y % n[1], x % n[0]]


def test_fused_stencils_reject_node_grids(cn):
    g = cn.Grid.Cartesian((2, 2, 2), (8, 8, 8), entity="node")
    out = cn.Grid.Cartesian((2, 2, 2), (8, 8, 8), entity="node")
    with pytest.raises(cn.CnError) as e:
        cn.ops.laplacian(g, out)
    assert "cell-centred" in str(e.value)
