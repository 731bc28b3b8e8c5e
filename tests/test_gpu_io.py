"""Grid <-> AoS file buffers on the device (cn_grid_to_aos / cn_grid_from_aos,
the block loops of IO::CartesianWriteHDF / CartesianReadHDF over Field2AOS /
AOS2Field) against the oracle (oracle/aos.py, itself pinned to the
reference's FieldAOS.h), bit for bit; a full-size round trip; the XDMF
writer and reader; HDF5 files of grids (CartesianWriteHDF / ReadHDF); error
behaviour."""
import ctypes as C
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from oracle import aos as A

pytestmark = pytest.mark.gpu
ENT = {0: "cell", 1: "node", 2: "face_x", 3: "face_y", 4: "face_z"}


def _span_case(rng, top):
    kind = rng.integers(0, 4)
    if kind == 0:
        return [0, 0, 0], list(top)
    if kind == 1:
        sb = [int(rng.integers(0, top[d])) for d in range(3)]
        return sb, [int(rng.integers(sb[d] + 1, top[d] + 1)) for d in range(3)]
    if kind == 2:
        return [int(rng.integers(-3, 2)) for d in range(3)], [int(rng.integers(top[d] - 1, top[d] + 4)) for d in range(3)]
    sb = [int(rng.integers(0, top[d])) for d in range(3)]
    se = [sb[d] + 1 for d in range(3)]
    if rng.random() < 0.5:
        sb[0], se[0] = top[0] + 1, top[0] + 3
    return sb, se


def _grid(cn, rng, entity, ncomp, dtype, nb, cells):
    g = cn.Grid.Cartesian(nb, cells, ncomp=ncomp, dtype=dtype, entity=ENT[entity])
    comps = []
    for c in range(ncomp):
        if np.dtype(dtype) == np.int32:
            a = rng.integers(-2**31, 2**31 - 1, size=g.comp_stride, dtype=np.int64).astype(np.int32)
        else:
            a = (rng.standard_normal(g.comp_stride) * 1e3).astype(dtype)
        g.upload(a, c)
        comps.append(a)
    return g, comps


# (grid, file) types; a floating-point value never lands in an int32 grid or file
CASES = [(np.float64, np.float64), (np.float64, np.float32), (np.float32, np.float32), (np.float32, np.float64),
         (np.int32, np.int32), (np.int32, np.float64), (np.int32, np.float32)]
READ_CASES = [(np.float64, np.float64), (np.float64, np.float32), (np.float32, np.float32), (np.float32, np.float64),
              (np.int32, np.int32), (np.float64, np.int32), (np.float32, np.int32)]


@pytest.mark.parametrize("grid_dtype,file_dtype", CASES)
def test_to_aos_matches_oracle(cn, grid_dtype, file_dtype):
    import torch
    rng = np.random.default_rng(CASES.index((grid_dtype, file_dtype)))
    for trial in range(12):
        entity = int(rng.choice([0, 0, 1, 2, 3, 4]))
        ncomp = int(rng.integers(1, 6)) if entity == 0 else int(rng.integers(1, 3))
        nb = [int(v) for v in rng.integers(1, 4, size=3)]
        cells = [int(v) for v in rng.integers(2, 9, size=3)]
        g, comps = _grid(cn, rng, entity, ncomp, grid_dtype, nb, cells)
        top = cn.IO.index_range(g)[1]
        sb, se = _span_case(rng, top)
        c0 = int(rng.integers(0, ncomp))
        nc = int(rng.integers(1, ncomp - c0 + 1))
        shape = (se[2] - sb[2], se[1] - sb[1], se[0] - sb[0], nc)
        init = np.full(shape, -5, dtype=file_dtype)
        out = torch.from_numpy(init.copy()).cuda()
        cn.IO.Field2AOS(g, (sb, se), file_dtype, comps=(c0, nc), out=out)
        torch.cuda.synchronize()
        want = A.grid_to_aos(comps[c0:c0 + nc], nb, cells, entity, g.block_stride, sb, se, init.copy().ravel())
        got = out.cpu().numpy().ravel()
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), (trial, entity, ncomp, c0, nc, sb, se)
        g.close()


@pytest.mark.parametrize("grid_dtype,file_dtype", READ_CASES)
def test_from_aos_matches_oracle(cn, grid_dtype, file_dtype):
    import torch
    rng = np.random.default_rng(100 + READ_CASES.index((grid_dtype, file_dtype)))
    for trial in range(12):
        entity = int(rng.choice([0, 0, 1, 2, 3, 4]))
        ncomp = int(rng.integers(1, 6)) if entity == 0 else int(rng.integers(1, 3))
        nb = [int(v) for v in rng.integers(1, 4, size=3)]
        cells = [int(v) for v in rng.integers(2, 9, size=3)]
        g, comps = _grid(cn, rng, entity, ncomp, grid_dtype, nb, cells)
        top = cn.IO.index_range(g)[1]
        sb, se = _span_case(rng, top)
        shape = (se[2] - sb[2], se[1] - sb[1], se[0] - sb[0], ncomp)
        if np.dtype(file_dtype) == np.int32:
            buf = rng.integers(-2**31, 2**31 - 1, size=shape, dtype=np.int64).astype(np.int32)
        else:
            buf = (rng.standard_normal(shape) * 1e5).astype(file_dtype)
        cn.IO.AOS2Field(torch.from_numpy(buf).cuda(), g, (sb, se))
        torch.cuda.synchronize()
        want = A.aos_to_grid(buf.ravel(), comps, nb, cells, entity, g.block_stride, sb, se)
        for c in range(ncomp):
            got = g.download(c)
            for flat, beg, ext in A._blocks(nb, cells, entity):
                n = ext[0] * ext[1] * ext[2]
                w = want[c][flat * g.block_stride: flat * g.block_stride + n]
                v = got[flat * g.block_stride: flat * g.block_stride + n]
                assert np.array_equal(v.view(np.uint8), w.view(np.uint8)), (trial, entity, c, flat)
        g.close()


def test_face_container_directions(cn):
    """A FaceContainer grid writes the face grid of the requested direction
    (AOSDriver<FaceContainer>, IO/FieldAOS.h:136-141)."""
    rng = np.random.default_rng(3)
    nb, cells = (2, 1, 3), (4, 5, 3)
    g = cn.Grid.Cartesian(nb, cells, ncomp=2, entity="face")
    for d in range(3):
        fg = g.faces[d]
        comps = []
        for c in range(2):
            a = rng.standard_normal(fg.comp_stride)
            g.upload(a, c, d)
            comps.append(a)
        b, e = cn.IO.index_range(g, face_dir=d)
        assert e == tuple(nb[k] * cells[k] + (k == d) for k in range(3))
        out = cn.IO.Field2AOS(g, face_dir=d).cpu().numpy()
        want = A.grid_to_aos(comps, nb, cells, 2 + d, fg.block_stride, b, e, np.zeros(out.size))
        assert np.array_equal(out.ravel(), want)
    g.close()


def test_full_size_round_trip(cn):
    """512^3 cells as 16^3 blocks of 32^3, 5 FP64 components: grid -> AoS ->
    fresh grid gives back every value, and the AoS buffer's per-component
    sums equal the grid's (a size-independent check of the gather)."""
    import torch
    nb, n = (16, 16, 16), (32, 32, 32)
    U = cn.Grid.Cartesian(nb, n, ncomp=5)
    cn.workloads.euler_pulse(U, seed=5)
    buf = cn.IO.Field2AOS(U)
    assert tuple(buf.shape) == (512, 512, 512, 5)
    for c in range(5):
        t = U.tensor(c)[:, : 32 ** 3]
        assert abs(float(buf[..., c].sum(dtype=torch.float64)) - float(t.sum(dtype=torch.float64))) <= \
            1e-9 * max(1.0, abs(float(t.sum(dtype=torch.float64))))
    V = cn.Grid.Cartesian(nb, n, ncomp=5)
    for c in range(5):
        V.tensor(c).zero_()
    cn.IO.AOS2Field(buf, V)
    torch.cuda.synchronize()
    for c in range(5):
        assert torch.equal(U.tensor(c)[:, : 32 ** 3], V.tensor(c)[:, : 32 ** 3])
    # one spot check of the layout: global cell (x, y, z) = (37, 5, 300)
    x, y, z = 37, 5, 300
    blk = (x // 32) + 16 * ((y // 32) + 16 * (z // 32))
    loc = (x % 32) + 32 * ((y % 32) + 32 * (z % 32))
    assert float(buf[z, y, x, 4]) == float(U.tensor(4)[blk, loc])
    del buf
    U.close()
    V.close()


def test_xdmf_write_read(cn, tmp_path, capsys):
    import torch
    rng = np.random.default_rng(9)
    nb, cells = (2, 3, 1), (4, 4, 6)
    g = cn.Grid.Cartesian(nb, cells, (0.0, -1.0, 2.0), (2.0, 2.0, 3.0), ncomp=3)
    comps = []
    for c in range(3):
        a = rng.standard_normal(g.comp_stride)
        g.upload(a, c)
        comps.append(a)
    fname = str(tmp_path / "velocity")
    cn.IO.CartesianWriteXDMF(fname, "U", g, time=0.25, file_dtype=np.float32)
    data = np.fromfile(fname + ".bin", dtype="<f4")
    b, e = cn.IO.index_range(g)
    want = A.grid_to_aos(comps, nb, cells, 0, g.block_stride, b, e, np.zeros(int(np.prod(e)) * 3, np.float32))
    assert np.array_equal(data, want)
    root = ET.parse(fname + ".xmf").getroot()
    topo = root.find("Domain/Grid/Topology")
    assert topo.get("TopologyType") == "3DCoRectMesh" and topo.get("Dimensions") == "7 13 9"
    org = [float(v) for v in root.find("Domain/Grid/Geometry/DataItem[@Name='Origin']").text.split()]
    assert org == [2.0, -1.0, 0.0]
    attr = root.find("Domain/Grid/Attribute")
    assert attr.get("Name") == "U" and attr.get("AttributeType") == "Vector" and attr.get("Center") == "Cell"
    item = attr.find("DataItem")
    assert item.get("Dimensions") == "6 12 8 3" and item.get("Precision") == "4" and item.get("Format") == "Binary"
    assert item.text.strip() == "./velocity.bin"
    # read back into a fresh grid (FP32 file -> FP64 grid)
    h = cn.Grid.Cartesian(nb, cells, ncomp=3)
    cn.IO.CartesianReadXDMF(fname, h, file_dtype=np.float32)
    torch.cuda.synchronize()
    for c in range(3):
        assert np.array_equal(h.download(c), A.aos_to_grid(data, [np.zeros(g.comp_stride)] * 3, nb, cells, 0,
                                                           g.block_stride, b, e)[c])
    g.close()
    h.close()


@pytest.mark.parametrize("entity,file_dtype", [(0, np.float64), (0, np.float32), (1, np.float64), (2, np.float32),
                                               (4, np.float64)])
def test_hdf_write_read(cn, tmp_path, capfd, entity, file_dtype):
    """CartesianWriteHDF: the HDF5 dataset "data" (z, y, x, components) equals
    the oracle's AoS buffer of the grid bit for bit, the XDMF wrapper points
    at it (cell and node data only); CartesianReadHDF restores the grid."""
    import torch
    rng = np.random.default_rng(40 + entity)
    nb, cells = (2, 1, 3), (4, 6, 4)
    ncomp = 3 if entity == 0 else 2
    g, comps = _grid(cn, rng, entity, ncomp, np.float64, nb, cells)
    fname = str(tmp_path / f"q{entity}")
    cn.IO.CartesianWriteHDF(fname, "q", g, time=1.5, file_dtype=file_dtype)
    torch.cuda.synchronize()
    b, e = cn.IO.index_range(g)
    shape, fdt = cn.IO.h5_query(fname + ".h5")
    assert shape == (e[2], e[1], e[0], ncomp) and fdt == np.dtype(file_dtype)
    data = cn.IO.h5_read(fname + ".h5")
    want = A.grid_to_aos(comps, nb, cells, entity, g.block_stride, b, e,
                         np.zeros(int(np.prod(e)) * ncomp, file_dtype))
    assert np.array_equal(data.ravel().view(np.uint8), want.view(np.uint8))
    out = capfd.readouterr().out
    mb = data.nbytes / 1024.0 / 1024.0
    assert f"CartesianWriteHDF: Allocating {mb:.1f} MB file buffer ({fname})" in out
    if entity in (0, 1):
        item = ET.parse(fname + ".xmf").getroot().find("Domain/Grid/Attribute/DataItem")
        assert item.get("Format") == "HDF" and item.text.strip() == f"./q{entity}.h5:/data"
        assert item.get("Dimensions") == f"{e[2]} {e[1]} {e[0]} {ncomp}"
    else:
        assert not os.path.exists(fname + ".xmf")  # no wrapper for face data (src/IO/HDFDriver.cpp:53-57)
    h = cn.Grid.Cartesian(nb, cells, ncomp=ncomp, entity=ENT[entity])
    cn.IO.CartesianReadHDF(fname, h, file_dtype=file_dtype)
    torch.cuda.synchronize()
    back = A.aos_to_grid(data.ravel(), [np.zeros(g.comp_stride)] * ncomp, nb, cells, entity, g.block_stride, b, e)
    for c in range(ncomp):
        assert np.array_equal(h.download(c), back[c])
    with pytest.raises(cn.CnError) as err:
        cn.IO.CartesianReadHDF(str(tmp_path / "none"), h)
    assert str(err.value) == f"CartesianReadHDF: File '{tmp_path / 'none'}' does not exist"
    g.close()
    h.close()


def test_errors(cn):
    import torch
    from cubismnova_b200 import _lib
    g = cn.Grid.Cartesian((2, 2, 2), (4, 4, 4), ncomp=2)
    buf = torch.zeros((8, 8, 8, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(cn.CnError):  # floating point -> int32
        cn.IO.Field2AOS(g, file_dtype=np.int32, out=buf)
    ig = cn.Grid.Cartesian((2, 2, 2), (4, 4, 4), dtype=np.int32)
    with pytest.raises(cn.CnError):  # floating point -> int32 grid
        cn.IO.AOS2Field(torch.zeros((8, 8, 8, 1), dtype=torch.float32, device="cuda"), ig)
    ig.close()
    with pytest.raises(cn.CnError):  # components outside the grid
        cn.IO.Field2AOS(g, comps=(1, 2))
    b = (C.c_int * 3)(0, 0, 0)
    e = (C.c_int * 3)(4, -1, 4)
    st = _lib.lib().cn_grid_to_aos(g.handle, 0, 1, b, e, 1, C.c_void_p(buf.data_ptr()), None)
    assert st == 1 and b"end before begin" in _lib.lib().cn_last_error_string()
    host = np.zeros(8 * 8 * 8, dtype=np.float64)  # pageable host memory: rejected before any launch
    st = _lib.lib().cn_grid_to_aos(g.handle, 0, 1, (C.c_int * 3)(0, 0, 0), (C.c_int * 3)(8, 8, 8), 1,
                                   C.c_void_p(host.ctypes.data), None)
    assert st == 1 and b"not device-accessible" in _lib.lib().cn_last_error_string()
    with pytest.raises(ValueError):
        cn.IO.Field2AOS(g, comps=(0, 1), out=torch.zeros((8, 8, 8, 1), dtype=torch.float64))
    big = cn.Grid.Cartesian((1, 1, 1), (4, 4, 4), ncomp=17)
    with pytest.raises(cn.CnError):  # more than 16 components in one call
        cn.IO.Field2AOS(big)
    cn.IO.Field2AOS(big, comps=(1, 16))  # 16 is fine
    torch.cuda.synchronize()
    g.close()
    big.close()
