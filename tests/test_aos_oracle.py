"""The AoS file-buffer oracle (oracle/aos.py) against the reference's own
Field2AOS / AOS2Field block loop (IO/FieldAOS.h, IO/CartesianHDF.h:76-80,
182-186) compiled here: cell, node and face grids, scalar and rank-1 cell
fields, FP64 and FP32 grids written as FP32 and FP64 files, file ranges that
cover the grid, cut it, reach past it or miss it.  Bit for bit, including
the buffer values outside the grid (left untouched by both)."""
import numpy as np
import pytest

import oracle as O
from oracle import aos as A

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference shim not built")


def _case(rng):
    entity = int(rng.choice([0, 0, 1, 2, 3, 4]))
    ncomp = 3 if (entity == 0 and rng.random() < 0.4) else 1
    nb = [int(v) for v in rng.integers(1, 4, size=3)]
    cells = [int(v) for v in rng.integers(2, 7, size=3)]
    grow = A.ENTITY_GROW[entity]
    top = [nb[d] * cells[d] + grow[d] for d in range(3)]
    kind = rng.integers(0, 4)
    if kind == 0:  # the whole grid
        sb, se_ = [0, 0, 0], top
    elif kind == 1:  # inside
        sb = [int(rng.integers(0, top[d])) for d in range(3)]
        se_ = [int(rng.integers(sb[d] + 1, top[d] + 1)) for d in range(3)]
    elif kind == 2:  # reaching past the grid on both sides
        sb = [int(rng.integers(-3, 2)) for d in range(3)]
        se_ = [int(rng.integers(top[d] - 1, top[d] + 4)) for d in range(3)]
    else:  # a slab one entity thick, or outside the grid in x
        sb = [int(rng.integers(0, top[d])) for d in range(3)]
        se_ = [sb[d] + 1 for d in range(3)]
        if rng.random() < 0.5:
            sb[0], se_[0] = top[0] + 1, top[0] + 3
    return entity, ncomp, nb, cells, sb, se_


@pytest.mark.parametrize("grid_dtype", [np.float64, np.float32])
@pytest.mark.parametrize("file_dtype", [np.float32, np.float64])
def test_field2aos_oracle_matches_reference(grid_dtype, file_dtype):
    rng = np.random.default_rng(11 + (grid_dtype == np.float32) + 2 * (file_dtype == np.float32))
    for trial in range(25):
        entity, ncomp, nb, cells, sb, se_ = _case(rng)
        stride = O.entity_stride(cells, entity, np.dtype(grid_dtype))
        nblk = int(np.prod(nb))
        data = (rng.standard_normal((ncomp, nblk * stride)) * 1e3).astype(grid_dtype)
        vol = int(np.prod([se_[d] - sb[d] for d in range(3)]))
        want = np.full(vol * ncomp, -7.5, dtype=file_dtype)
        got = want.copy()
        A.grid_to_aos(list(data), nb, cells, entity, stride, sb, se_, want)
        O.ref_field_aos(data, nb, cells, entity, stride, sb, se_, file_dtype, got, to_aos=True)
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), (trial, entity, ncomp, nb, cells, sb, se_)


@pytest.mark.parametrize("grid_dtype", [np.float64, np.float32])
@pytest.mark.parametrize("file_dtype", [np.float32, np.float64])
def test_aos2field_oracle_matches_reference(grid_dtype, file_dtype):
    rng = np.random.default_rng(23 + (grid_dtype == np.float32) + 2 * (file_dtype == np.float32))
    for trial in range(25):
        entity, ncomp, nb, cells, sb, se_ = _case(rng)
        stride = O.entity_stride(cells, entity, np.dtype(grid_dtype))
        nblk = int(np.prod(nb))
        data = (rng.standard_normal((ncomp, nblk * stride)) * 1e3).astype(grid_dtype)
        vol = int(np.prod([se_[d] - sb[d] for d in range(3)]))
        buf = (rng.standard_normal(vol * ncomp) * 1e5).astype(file_dtype)
        want = A.aos_to_grid(buf, list(data), nb, cells, entity, stride, sb, se_)
        _, got = O.ref_field_aos(data, nb, cells, entity, stride, sb, se_, file_dtype, buf, to_aos=False)
        # compare each block's own extent (the padding past it is not data)
        for flat, beg, ext in A._blocks(nb, cells, entity):
            n = ext[0] * ext[1] * ext[2]
            for c in range(ncomp):
                g = got[c][flat * stride: flat * stride + n]
                w = want[c][flat * stride: flat * stride + n]
                assert np.array_equal(g.view(np.uint8), w.view(np.uint8)), (trial, entity, flat, c)


def test_reference_face_container_read_is_the_face_field_read():
    """AOSDriver<FaceContainer>::read (IO/FieldAOS.h:143-148) passes the face
    field where the buffer goes and does not compile; the shim reads through
    the face field of the direction.  A write followed by that read restores
    every face value of the range (the round trip the container means)."""
    rng = np.random.default_rng(5)
    nb, cells = [2, 2, 1], [3, 4, 5]
    for entity in (2, 3, 4):
        stride = O.entity_stride(cells, entity, np.dtype(np.float64))
        data = rng.standard_normal((1, 4 * stride))
        top = [nb[d] * cells[d] + A.ENTITY_GROW[entity][d] for d in range(3)]
        buf = np.zeros(int(np.prod(top)), dtype=np.float64)
        O.ref_field_aos(data, nb, cells, entity, stride, [0, 0, 0], top, np.float64, buf, to_aos=True)
        _, back = O.ref_field_aos(np.zeros_like(data), nb, cells, entity, stride, [0, 0, 0], top, np.float64, buf,
                                  to_aos=False)
        for flat, beg, ext in A._blocks(nb, cells, entity):
            n = ext[0] * ext[1] * ext[2]
            assert np.array_equal(back[0][flat * stride: flat * stride + n], data[0][flat * stride: flat * stride + n])
