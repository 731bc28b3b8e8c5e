"""IO: grids to and from array-of-structures (AoS) file buffers on the GPU.

The reference writes a grid by gathering every block field into one AoS
buffer on the host (IO/CartesianHDF.h:76-80, Field2AOS of IO/FieldAOS.h) and
hands it to HDF5 (src/IO/HDFDriver.cpp: dataset "data" of dims
(z, y, x, components)) with an XDMF wrapper (IO/XDMFDriver.h).  Here the
gather (and the scatter of the read) is one kernel over the whole grid
(``cn_grid_to_aos`` / ``cn_grid_from_aos``); the buffer is a CUDA tensor of
shape (z, y, x, components).

No HDF5 library is part of this build, so ``CartesianWriteHDF`` and
``CartesianReadHDF`` behave as the reference built without HDF
(``CUBISM_USE_HDF`` undefined, IO/CartesianHDF.h:92-95, 188-191): they print
"HDF not supported" and return.  ``CartesianWriteXDMF`` / ``CartesianReadXDMF``
write and read the same dataset as a raw little-endian binary file with the
reference's XDMF wrapper pointing at it (``Format="Binary"`` instead of
``"HDF"``), which XDMF readers open directly.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

from . import _lib
from .grid import _DT, FaceCartesian, _stream_handle

_GROW = {"cell": (0, 0, 0), "node": (1, 1, 1), "face_x": (1, 0, 0), "face_y": (0, 1, 0), "face_z": (0, 0, 1)}
_NP_OF_TORCH = {}


def _scalar_grid(grid, face_dir):
    """The grid holding the values: a face container's face grid of one
    direction (AOSDriver<FaceContainer>, IO/FieldAOS.h:136-149)."""
    if isinstance(grid, FaceCartesian):
        return grid.faces[int(face_dir)]
    return grid


def index_range(grid, face_dir=0):
    """Global entity index range [begin, end) of a grid's values: cells, or
    cells + 1 along grown dimensions (the file span of a whole-grid write:
    IO/CartesianHDF.h:63-69 with the grid's global mesh)."""
    g = _scalar_grid(grid, face_dir)
    nb, cells, grow = g.getSize(), g.getBlockCells(), _GROW[g.entity]
    return (0, 0, 0), tuple(nb[d] * cells[d] + grow[d] for d in range(3))


def _span(grid, span, face_dir):
    if span is None:
        return index_range(grid, face_dir)
    b, e = span
    b, e = tuple(int(v) for v in b), tuple(int(v) for v in e)
    if any(e[d] < b[d] for d in range(3)):
        raise ValueError("file range end before begin")
    return b, e


def _torch_dtype(dt):
    import torch
    m = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32, np.dtype(np.int32): torch.int32}
    if not _NP_OF_TORCH:
        _NP_OF_TORCH.update({v: k for k, v in m.items()})
    return m[np.dtype(dt)]


def _np_dtype(torch_dtype):
    _torch_dtype(np.float64)
    if torch_dtype not in _NP_OF_TORCH:
        raise ValueError(f"unsupported buffer dtype {torch_dtype}")
    return _NP_OF_TORCH[torch_dtype]


def Field2AOS(grid, span=None, file_dtype=None, comps=None, out=None, face_dir=0, stream=None):
    """Device AoS buffer of a grid (IO/FieldAOS.h:186-194 over every block).

    ``span``: ((bx, by, bz), (ex, ey, ez)) global entity index range of the
    file (default: the whole grid); ``file_dtype``: float64 / float32 / int32
    (default: the grid's); ``comps``: (first, count) of the components
    (default: all); ``out``: an existing CUDA tensor to write into (points
    of the range outside the grid keep its values; a new buffer is zeroed).
    Returns the tensor, shape (z, y, x, count)."""
    import torch
    g = _scalar_grid(grid, face_dir)
    b, e = _span(grid, span, face_dir)
    fdt = np.dtype(file_dtype or g.dtype)
    c0, nc = comps if comps is not None else (0, g.ncomp)
    shape = (e[2] - b[2], e[1] - b[1], e[0] - b[0], nc)
    if out is None:
        out = torch.zeros(shape, dtype=_torch_dtype(fdt), device="cuda")
    elif (tuple(out.shape) != shape or out.dtype != _torch_dtype(fdt) or not out.is_contiguous()
          or not out.is_cuda):
        raise ValueError(f"Field2AOS: out must be a contiguous CUDA {fdt} tensor of shape {shape}")
    _lib.check(_lib.lib().cn_grid_to_aos(g.handle, int(c0), int(nc), _lib.ivec3(b), _lib.ivec3(e), _DT[fdt],
                                         C.c_void_p(out.data_ptr()), _stream_handle(stream)))
    return out


def AOS2Field(buf, grid, span=None, comps=None, face_dir=0, stream=None):
    """Reads a device AoS buffer (shape (z, y, x, count) of the range) into
    the grid (IO/FieldAOS.h:196-206 over every block); grid values outside
    the range are unchanged."""
    g = _scalar_grid(grid, face_dir)
    b, e = _span(grid, span, face_dir)
    c0, nc = comps if comps is not None else (0, g.ncomp)
    shape = (e[2] - b[2], e[1] - b[1], e[0] - b[0], nc)
    fdt = _np_dtype(buf.dtype)
    if tuple(buf.shape) != shape or not buf.is_contiguous() or not buf.is_cuda:
        raise ValueError(f"AOS2Field: buf must be a contiguous CUDA tensor of shape {shape}")
    _lib.check(_lib.lib().cn_grid_from_aos(g.handle, int(c0), int(nc), _lib.ivec3(b), _lib.ivec3(e), _DT[fdt],
                                           C.c_void_p(buf.data_ptr()), _stream_handle(stream)))


def CartesianWriteHDF(fname, aname, grid, time=0.0, face_dir=0, create_xdmf=True, file_dtype=None, span=None):
    """IO::CartesianWriteHDF (IO/CartesianHDF.h:42-96, 113-131) of a build without
    HDF5: prints the reference's message and writes nothing."""
    sys.stderr.write(f"CartesianWriteHDF: HDF not supported ({fname})\n")


def CartesianReadHDF(fname, grid, face_dir=0, file_dtype=None, span=None):
    """IO::CartesianReadHDF (IO/CartesianHDF.h:147-192, 206-220) of a build without
    HDF5: prints the reference's message and reads nothing."""
    sys.stderr.write(f"CartesianReadHDF: HDF not supported ({fname})\n")


def _xdmf(fname, aname, g, b, e, nc, fdt, time):
    """XDMF wrapper of IO/XDMFDriver.h:31-160 (uniform mesh, cell or node
    data) for the dataset in fname.bin."""
    dims = 3
    h = g.getCellSize()
    origin = getattr(g, "_begin", (0.0, 0.0, 0.0))
    node = g.entity == "node"
    ext = [e[d] - b[d] for d in range(3)]
    # the mesh of the range: its cells (nodes minus one for node data)
    mesh_nodes = [ext[d] if node else ext[d] + 1 for d in range(3)]
    org = [origin[d] + b[d] * h[d] for d in range(3)]
    attr = "Scalar" if nc == 1 else ("Vector" if nc == dims else "Tensor")
    ntype = "Int" if fdt == np.dtype(np.int32) else "Float"
    zyx = lambda v: " ".join(str(v[2 - i]) for i in range(3))
    fmt = lambda v: " ".join(repr(float(v[2 - i])) for i in range(3))
    base = os.path.basename(fname)
    lines = [
        '<?xml version="1.0" ?>',
        '<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>',
        '<Xdmf Version="2.0">',
        "<Domain>",
        '\t<Grid GridType="Uniform">',
        f'\t\t<Time Value="{time:e}"/>',
        "",
        f'\t\t<Topology TopologyType="3DCoRectMesh" Dimensions="{zyx(mesh_nodes)}"/>',
        "",
        '\t\t<Geometry GeometryType="Origin_DxDyDz">',
        '\t\t\t<DataItem Name="Origin" Dimensions="3" NumberType="Float" Precision="8" Format="XML">',
        f"\t\t\t\t{fmt(org)}",
        "\t\t\t</DataItem>",
        '\t\t\t<DataItem Name="Spacing" Dimensions="3" NumberType="Float" Precision="8" Format="XML">',
        f"\t\t\t\t{fmt(h)}",
        "\t\t\t</DataItem>",
        "\t\t</Geometry>",
        "",
        f'\t\t<Attribute Name="{aname}" AttributeType="{attr}" Center="{"Node" if node else "Cell"}">',
        f'\t\t\t<DataItem Dimensions="{zyx(ext)} {nc}" NumberType="{ntype}" Precision="{fdt.itemsize}" '
        f'Format="Binary" Endian="Little">',
        f"\t\t\t\t./{base}.bin",
        "\t\t\t</DataItem>",
        "\t\t</Attribute>",
        "\t</Grid>",
        "</Domain>",
        "</Xdmf>",
    ]
    with open(fname + ".xmf", "w") as f:
        f.write("\n".join(lines) + "\n")


def CartesianWriteXDMF(fname, aname, grid, time=0.0, face_dir=0, create_xdmf=True, file_dtype=None, span=None,
                       stream=None):
    """The dataset of CartesianWriteHDF (dims (z, y, x, components) of
    ``file_dtype``, default the grid's) as ``fname.bin`` (raw,
    little-endian) plus ``fname.xmf``; face data gets no XDMF wrapper, as in
    the reference (src/IO/HDFDriver.cpp:53-57).  The gather runs on the GPU;
    the buffer comes to pinned host memory in one copy."""
    import torch
    g = _scalar_grid(grid, face_dir)
    b, e = _span(grid, span, face_dir)
    fdt = np.dtype(file_dtype or g.dtype)
    s = stream or torch.cuda.current_stream()
    with torch.cuda.stream(s):
        dev = Field2AOS(grid, (b, e), fdt, face_dir=face_dir, stream=s)
        host = torch.empty(dev.shape, dtype=dev.dtype, pin_memory=True)
        host.copy_(dev, non_blocking=True)
    s.synchronize()
    host.numpy().astype(fdt.newbyteorder("<"), copy=False).tofile(fname + ".bin")
    if create_xdmf and not g.entity.startswith("face"):
        _xdmf(fname, aname, g, b, e, dev.shape[3], fdt, time)


def CartesianReadXDMF(fname, grid, face_dir=0, file_dtype=None, span=None, stream=None):
    """Reads ``fname.bin`` written by CartesianWriteXDMF for the same range
    and file type into the grid."""
    import torch
    g = _scalar_grid(grid, face_dir)
    b, e = _span(grid, span, face_dir)
    fdt = np.dtype(file_dtype or g.dtype)
    shape = (e[2] - b[2], e[1] - b[1], e[0] - b[0], g.ncomp)
    path = fname + ".bin"
    if not os.path.exists(path):
        raise RuntimeError(f"CartesianReadXDMF: File '{fname}' does not exist")
    host = np.fromfile(path, dtype=fdt.newbyteorder("<"))
    if host.size != int(np.prod(shape)):
        raise ValueError(f"CartesianReadXDMF: '{path}' holds {host.size} values, the range needs {int(np.prod(shape))}")
    s = stream or torch.cuda.current_stream()
    with torch.cuda.stream(s):
        dev = torch.from_numpy(host.astype(fdt).reshape(shape)).pin_memory().to("cuda", non_blocking=True)
        AOS2Field(dev, grid, (b, e), face_dir=face_dir, stream=s)
    s.synchronize()
