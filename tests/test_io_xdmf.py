"""The XDMF wrapper of CartesianWriteXDMF (the structure of IO/XDMFDriver.h:31-160
with a raw binary data item), written for stub grids on the CPU: cell and
node centring, file ranges, attribute types."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from cubismnova_b200 import io as IO


class _Grid:
    def __init__(self, entity, h, begin):
        self.entity, self._h, self._begin = entity, h, begin

    def getCellSize(self):
        return self._h


def _parse(path):
    root = ET.parse(path).getroot()
    g = root.find("Domain/Grid")
    topo = g.find("Topology").get("Dimensions")
    org = [float(v) for v in g.find("Geometry/DataItem[@Name='Origin']").text.split()]
    sp = [float(v) for v in g.find("Geometry/DataItem[@Name='Spacing']").text.split()]
    attr = g.find("Attribute")
    item = attr.find("DataItem")
    return dict(time=float(g.find("Time").get("Value")), topo=topo, org=org, sp=sp, name=attr.get("Name"),
                type=attr.get("AttributeType"), center=attr.get("Center"), dims=item.get("Dimensions"),
                ntype=item.get("NumberType"), prec=item.get("Precision"), fmt=item.get("Format"),
                endian=item.get("Endian"), file=item.text.strip())


def test_cell_data_whole_grid(tmp_path):
    g = _Grid("cell", (0.5, 0.25, 0.125), (1.0, 2.0, 3.0))
    IO._xdmf(str(tmp_path / "rho"), "rho", g, (0, 0, 0), (8, 4, 2), 1, np.dtype(np.float32), 1.5)
    x = _parse(tmp_path / "rho.xmf")
    assert x["time"] == 1.5 and x["name"] == "rho" and x["type"] == "Scalar" and x["center"] == "Cell"
    assert x["topo"] == "3 5 9"  # nodes z, y, x
    assert x["org"] == [3.0, 2.0, 1.0] and x["sp"] == [0.125, 0.25, 0.5]
    assert x["dims"] == "2 4 8 1" and x["ntype"] == "Float" and x["prec"] == "4"
    assert x["fmt"] == "Binary" and x["endian"] == "Little" and x["file"] == "./rho.bin"


def test_node_data_subrange_and_types(tmp_path):
    g = _Grid("node", (0.5, 0.5, 0.5), (0.0, 0.0, 0.0))
    # nodes [2, 5) x [1, 4) x [0, 3): a 2^3-cell sub-mesh starting at node (2, 1, 0)
    IO._xdmf(str(tmp_path / "u"), "u", g, (2, 1, 0), (5, 4, 3), 3, np.dtype(np.float64), 0.0)
    x = _parse(tmp_path / "u.xmf")
    assert x["center"] == "Node" and x["type"] == "Vector"
    assert x["topo"] == "3 3 3" and x["dims"] == "3 3 3 3"
    assert x["org"] == [0.0, 0.5, 1.0] and x["prec"] == "8"
    IO._xdmf(str(tmp_path / "t"), "t", _Grid("cell", (1.0, 1.0, 1.0), (0.0, 0.0, 0.0)), (0, 0, 0), (2, 2, 2), 9,
             np.dtype(np.int32), 0.0)
    x = _parse(tmp_path / "t.xmf")
    assert x["type"] == "Tensor" and x["ntype"] == "Int" and x["prec"] == "4" and x["dims"] == "2 2 2 9"


def test_hdf_wrapper_points_at_the_dataset(tmp_path):
    """Format="HDF" and "./basename.h5:/data", as IO/XDMFDriver.h:155-156."""
    g = _Grid("cell", (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    IO._xdmf(str(tmp_path / "p"), "p", g, (0, 0, 0), (4, 4, 4), 1, np.dtype(np.float64), 2.0, fmt="HDF")
    x = _parse(tmp_path / "p.xmf")
    assert x["fmt"] == "HDF" and x["file"] == "./p.h5:/data" and x["endian"] is None
    assert x["dims"] == "4 4 4 1" and x["prec"] == "8" and x["time"] == 2.0


def test_face_data_gets_no_wrapper(tmp_path):
    from cubismnova_b200 import _lib
    g = _Grid("face_x", (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    IO._ENTITY_CODE["face_x"] = 2
    try:
        with pytest.raises(_lib.CnError) as e:
            IO._xdmf(str(tmp_path / "f"), "f", g, (0, 0, 0), (2, 2, 2), 1, np.dtype(np.float64), 0.0)
        assert e.value.status == 12
    finally:
        del IO._ENTITY_CODE["face_x"]


class _Topo:
    def __init__(self, entity, nb, cells):
        self.entity, self._nb, self._cells = entity, nb, cells

    def getSize(self):
        return self._nb

    def getBlockCells(self):
        return self._cells


def test_whole_grid_file_range_per_entity():
    """The file range of a whole-grid write (IO/CartesianHDF.h:63-69 with the
    global mesh): cells, or cells + 1 along grown dimensions."""
    nb, cells = (2, 3, 4), (5, 6, 7)
    want = {"cell": (10, 18, 28), "node": (11, 19, 29), "face_x": (11, 18, 28), "face_y": (10, 19, 28),
            "face_z": (10, 18, 29)}
    for ent, e in want.items():
        assert IO.index_range(_Topo(ent, nb, cells)) == ((0, 0, 0), e)


def test_file_range_validation():
    g = _Topo("cell", (1, 1, 1), (4, 4, 4))
    assert IO._span(g, None, 0) == ((0, 0, 0), (4, 4, 4))
    assert IO._span(g, ((-1, 0, 2), (5, 4, 2)), 0) == ((-1, 0, 2), (5, 4, 2))  # empty z extent is allowed
    try:
        IO._span(g, ((0, 0, 0), (4, -1, 4)), 0)
        raise AssertionError("end before begin accepted")
    except ValueError as e:
        assert "end before begin" in str(e)
