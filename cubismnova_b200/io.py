"""IO: grids to and from array-of-structures (AoS) file buffers on the GPU,
HDF5 container files and their XDMF wrappers.

The reference writes a grid by gathering every block field into one AoS
buffer on the host (IO/CartesianHDF.h:76-80, Field2AOS of IO/FieldAOS.h) and
hands it to HDF5 (src/IO/HDFDriver.cpp: dataset "data" of dims
(z, y, x, components)) with an XDMF wrapper (IO/XDMFDriver.h).  Here the
gather (and the scatter of the read) is one kernel over the whole grid
(``cn_grid_to_aos`` / ``cn_grid_from_aos``); the buffer is a CUDA tensor of
shape (z, y, x, components).

``CartesianWriteHDF`` / ``CartesianReadHDF`` write and read that dataset in
an HDF5 file (``fname.h5``) and the reference's XDMF wrapper
(``Format="HDF"``).  The library lays the HDF5 file out itself, from the
published file-format specification (no libhdf5 in this build): superblock
version 0, an old-style root group, version 1 object headers, the data
contiguous.  ``h5_write`` / ``h5_query`` / ``h5_read`` are the host-side file
calls (no GPU).  ``CartesianWriteXDMF`` / ``CartesianReadXDMF`` keep the
dataset as a raw little-endian binary file beside the same wrapper
(``Format="Binary"``).
"""
from __future__ import annotations

import ctypes as C
import os

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


_DT_OF_CODE = {v: k for k, v in _DT.items()}


def h5_write(path, array, dataset="data", chunked=False):
    """Writes a host array (float64, float32 or int32) as dataset ``dataset``
    of an HDF5 file (root group); ``chunked``: one chunk over the dataset, the
    layout the reference's ``H5Pset_chunk(dims)`` gives (under 4 GiB)."""
    a = np.ascontiguousarray(array)
    if a.dtype.newbyteorder("=") not in _DT or a.ndim < 1:
        raise ValueError(f"h5_write: float64, float32 or int32 arrays of rank >= 1, not {a.dtype} rank {a.ndim}")
    a = a.astype(a.dtype.newbyteorder("<"), copy=False)
    dims = (C.c_longlong * a.ndim)(*a.shape)
    _lib.check(_lib.lib().cn_h5_write(os.fsencode(path), dataset.encode(), a.ndim, dims,
                                      _DT[np.dtype(a.dtype.newbyteorder("="))], C.c_void_p(a.ctypes.data),
                                      int(bool(chunked))))


def h5_query(path, dataset="data"):
    """(shape, dtype) of a dataset in the root group of an HDF5 file."""
    rank, dt = C.c_int(), C.c_int()
    dims = (C.c_longlong * 32)()
    _lib.check(_lib.lib().cn_h5_query(os.fsencode(path), dataset.encode(), C.byref(rank), dims, C.byref(dt)))
    return tuple(int(dims[i]) for i in range(rank.value)), _DT_OF_CODE[dt.value]


def h5_read(path, dataset="data", count=None, dtype=None):
    """The hyperslab [0, count) (default: the whole dataset) of a dataset as a
    host array of ``dtype`` (default: the file's)."""
    shape, fdt = h5_query(path, dataset)
    cnt = tuple(shape if count is None else (int(c) for c in count))
    out = np.empty(cnt, dtype=np.dtype(dtype or fdt))
    if out.dtype not in _DT:
        raise ValueError(f"h5_read: float64, float32 or int32 output, not {out.dtype}")
    _lib.check(_lib.lib().cn_h5_read(os.fsencode(path), dataset.encode(), len(cnt), (C.c_longlong * len(cnt))(*cnt),
                                     _DT[out.dtype], C.c_void_p(out.ctypes.data)))
    return out


def CartesianWriteHDF(fname, aname, grid, time=0.0, face_dir=0, create_xdmf=True, file_dtype=None, span=None,
                      stream=None):
    """IO::CartesianWriteHDF (IO/CartesianHDF.h:42-96, 113-131 with
    src/IO/HDFDriver.cpp:25-111): the grid's values on the file range
    ``span`` (default: the whole grid) as dataset "data" of dims
    (z, y, x, components) and type ``file_dtype`` (default: the grid's) in
    ``fname.h5``, plus ``fname.xmf`` for cell and node data when
    ``create_xdmf``.  Gathered on the GPU in one kernel, copied down once."""
    g = _scalar_grid(grid, face_dir)
    b, e = _span(grid, span, face_dir)
    fdt = np.dtype(file_dtype or g.dtype)
    _lib.check(_lib.lib().cn_grid_write_hdf(g.handle, os.fsencode(fname), aname.encode(), 0, g.ncomp,
                                            _lib.ivec3(b), _lib.ivec3(e), _DT[fdt], float(time),
                                            int(bool(create_xdmf)), _stream_handle(stream)))


def CartesianReadHDF(fname, grid, face_dir=0, file_dtype=None, span=None, stream=None):
    """IO::CartesianReadHDF (IO/CartesianHDF.h:147-192, 206-220 with
    src/IO/HDFDriver.cpp:113-165): the hyperslab [0, count) of dataset
    "data" in ``fname.h5`` (count: the range's extent and the grid's
    components) into the grid's file range; a missing file raises the
    reference's "CartesianReadHDF: File 'fname' does not exist"."""
    g = _scalar_grid(grid, face_dir)
    b, e = _span(grid, span, face_dir)
    fdt = np.dtype(file_dtype or g.dtype)
    _lib.check(_lib.lib().cn_grid_read_hdf(g.handle, os.fsencode(fname), 0, g.ncomp, _lib.ivec3(b), _lib.ivec3(e),
                                           _DT[fdt], _stream_handle(stream)))


_ENTITY_CODE = {"cell": 0, "node": 1}


def _xdmf(fname, aname, g, b, e, nc, fdt, time, fmt="Binary"):
    """XDMF wrapper of IO/XDMFDriver.h:31-160 (uniform mesh, cell or node
    data, ``cn_xdmf_write``) for the dataset in fname.bin (``fmt`` "Binary")
    or fname.h5:/data ("HDF")."""
    h = (C.c_double * 3)(*[float(v) for v in g.getCellSize()])
    origin = (C.c_double * 3)(*[float(v) for v in getattr(g, "_begin", (0.0, 0.0, 0.0))])
    _lib.check(_lib.lib().cn_xdmf_write(os.fsencode(fname), aname.encode(), _ENTITY_CODE[g.entity], _lib.ivec3(b),
                                        _lib.ivec3(e), origin, h, int(nc), _DT[np.dtype(fdt)], float(time),
                                        0 if fmt == "HDF" else 1))


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
