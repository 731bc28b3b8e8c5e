"""Grid::Cartesian on one GPU (include/Cubism/Grid/Cartesian.h).

All blocks of all components stay resident in HBM in the reference layout
(component-major, block-major, x fastest, 32-byte padded blocks), so a host
array in the reference's SoA order uploads with one copy and
``Cartesian.loadLab`` becomes an on-device gather.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .core import IndexRange

_DT = {np.dtype(np.float32): _lib.CN_FLOAT32, np.dtype(np.float64): _lib.CN_FLOAT64,
       np.dtype(np.int32): _lib.CN_INT32}
# Cubism::EntityType of the values (cn_entity)
ENTITIES = {"cell": 0, "node": 1, "face_x": 2, "face_y": 3, "face_z": 4}


def _stream_handle(stream):
    """cudaStream_t of a torch stream (or the current torch stream)."""
    if stream is None:
        import torch
        if torch.cuda.is_available():
            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


class BCVector:
    """The BC vector of one block field (Block/Field.h:73-74, 437-442).

    ``push_back`` appends on the device table as well; order is preserved
    and matters exactly as in the reference."""

    def __init__(self, grid, comp, block):
        self._g, self._c, self._b = grid, comp, block

    def _list(self):
        return self._g._bcs[self._c].setdefault(self._b, [])

    def push_back(self, bc):
        info = bc.getBoundaryInfo()
        _lib.check(_lib.lib().cn_bc_push(self._g._h, self._c, self._b, info.dir, info.side,
                                         bc.kind, C.c_double(bc.value)))
        self._list().append(bc)

    append = push_back

    def clear(self):
        _lib.check(_lib.lib().cn_bc_clear(self._g._h, self._c, self._b))
        self._list().clear()

    def __len__(self):
        return len(self._list())

    def __iter__(self):
        return iter(list(self._list()))

    def __getitem__(self, i):
        return self._list()[i]


class FieldState:
    """Cartesian::FieldState (Grid/Cartesian.h:78-85) without the mesh pointer."""

    def __init__(self, block_index):
        self.block_index = block_index


class BlockField:
    """Non-owning view of one scalar block field (component ``comp``)."""

    def __init__(self, grid, flat, comp):
        self._g, self.flat, self.comp = grid, flat, comp
        nb = grid.getSize()
        self._state = FieldState((flat % nb[0], (flat // nb[0]) % nb[1], flat // (nb[0] * nb[1])))

    def getState(self):
        return self._state

    def getIndexRange(self):
        return IndexRange(self._g.block_extent(self.flat))

    def getBC(self):
        return BCVector(self._g, self.comp, self.flat)

    @property
    def grid(self):
        return self._g


class TensorBlock:
    """Rank-1 block (component access ``[c]``), FieldContainer-like."""

    def __init__(self, grid, flat):
        self._g, self.flat = grid, flat

    def __getitem__(self, c):
        if not 0 <= c < self._g.ncomp:
            raise IndexError("component out of range")
        return BlockField(self._g, self.flat, c)

    def getState(self):
        return BlockField(self._g, self.flat, 0).getState()

    def getIndexRange(self):
        return IndexRange(self._g.block_extent(self.flat))


class Cartesian:
    """Grid::Cartesian(nblocks, block_cells, begin, end) with ``ncomp`` components.

    ``entity`` is the Cubism::EntityType of the values: "cell" (default),
    "node", one direction of a face container ("face_x", "face_y",
    "face_z"), or "face" for the whole container (a ``FaceCartesian``);
    ``getBlockCells`` is the mesh, ``getBlockExtent`` the values per block
    (cells + 1 for nodes and along the face direction)."""

    def __new__(cls, *args, **kwargs):
        entity = kwargs.get("entity", args[6] if len(args) > 6 else "cell")
        if entity == "face":
            kw = {k: v for k, v in kwargs.items() if k != "entity"}
            return FaceCartesian(*args[:6], **kw)
        return super().__new__(cls)

    def __init__(self, nblocks, block_cells, begin=(0.0, 0.0, 0.0), end=(1.0, 1.0, 1.0),
                 ncomp: int = 1, dtype=np.float64, entity: str = "cell"):
        nb = tuple(int(v) for v in (nblocks if hasattr(nblocks, "__len__") else (nblocks,) * 3))
        bc = tuple(int(v) for v in (block_cells if hasattr(block_cells, "__len__") else (block_cells,) * 3))
        self.dtype = np.dtype(dtype)
        if self.dtype not in _DT:
            raise ValueError("dtype must be float32, float64 or int32")
        self.ncomp = int(ncomp)
        h = C.c_void_p()
        self.entity = entity
        self._begin = tuple(float(v) for v in begin)
        self._end = tuple(float(v) for v in end)
        _lib.check(_lib.lib().cn_grid_create_entity(_lib.ivec3(nb), _lib.ivec3(bc), self.ncomp, _DT[self.dtype],
                                                    ENTITIES[entity], _lib.dvec3(begin), _lib.dvec3(end),
                                                    C.byref(h)))
        self._h = h
        info = (C.c_int * 8)()
        _lib.check(_lib.lib().cn_grid_shape(h, info))
        self._nb, self._n, self._cells = nb, tuple(info[3:6]), bc
        self._bcs = [dict() for _ in range(self.ncomp)]
        bs, cs, tb = C.c_int64(), C.c_int64(), C.c_size_t()
        _lib.check(_lib.lib().cn_grid_layout(h, C.byref(bs), C.byref(cs), C.byref(tb)))
        self.block_stride, self.comp_stride, self.total_bytes = bs.value, cs.value, tb.value

    @classmethod
    def view_of(cls, handle, owner=None):
        """Non-owning Python view of a grid created inside the library (for
        example a multigrid level); ``owner`` is kept alive with the view."""
        g = cls.__new__(cls)
        g._h = C.c_void_p(handle.value if isinstance(handle, C.c_void_p) else handle)
        g._owned = False
        g._owner = owner
        bs, cs, tb = C.c_int64(), C.c_int64(), C.c_size_t()
        _lib.check(_lib.lib().cn_grid_layout(g._h, C.byref(bs), C.byref(cs), C.byref(tb)))
        g.block_stride, g.comp_stride, g.total_bytes = bs.value, cs.value, tb.value
        info = (C.c_int * 8)()
        _lib.check(_lib.lib().cn_grid_shape(g._h, info))
        g._nb, g._n = tuple(info[0:3]), tuple(info[3:6])
        ent, cells = C.c_int(), (C.c_int * 3)()
        _lib.check(_lib.lib().cn_grid_entity(g._h, C.byref(ent), cells))
        g.entity = {v: k for k, v in ENTITIES.items()}[ent.value]
        g._cells = tuple(cells)
        g.ncomp = info[6]
        g.dtype = {v: k for k, v in _DT.items()}[info[7]]
        g._bcs = [dict() for _ in range(g.ncomp)]
        return g

    # -- lifetime
    def close(self):
        if getattr(self, "_owned", True) and getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().cn_grid_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- topology (Grid/Cartesian.h:230-274)
    def size(self):
        return self._nb[0] * self._nb[1] * self._nb[2]

    def getSize(self):
        return self._nb

    def getBlockCells(self):
        """Cells per block of the mesh (Grid/Cartesian.h:240-256)."""
        return self._cells

    def getBlockExtent(self):
        """Values per block and direction of the largest block field (cells,
        or cells + 1 for nodes / along a face direction); the storage and lab
        strides of every block follow it."""
        return self._n

    def block_extent(self, flat):
        """Index-range extent of block field ``flat``: node and face fields
        hold cells + 1 entities along a grown direction only in the last block
        of that direction (Grid/BlockFieldAssembler.h:124-135)."""
        flat = self.flat_index(flat)
        bi = (flat % self._nb[0], (flat // self._nb[0]) % self._nb[1], flat // (self._nb[0] * self._nb[1]))
        cells = self.getBlockCells()
        return tuple(self._n[d] if bi[d] == self._nb[d] - 1 else min(self._n[d], cells[d]) for d in range(3))

    def getCellSize(self):
        h = (C.c_double * 3)()
        _lib.check(_lib.lib().cn_grid_cell_size(self._h, h))
        return tuple(h)

    def device_error(self, clear: bool = True) -> int:
        """The grid's device error word (cn_grid_device_error): 0, or the code
        a kernel recorded when it gave up a bounded wait; waits for the device
        and, with clear, resets the word."""
        w = C.c_int()
        _lib.check(_lib.lib().cn_grid_device_error(self._h, C.byref(w), 1 if clear else 0))
        return w.value

    def flat_index(self, p):
        if isinstance(p, (int, np.integer)):
            if not 0 <= int(p) < self.size():
                raise IndexError("block index out of range")
            return int(p)
        x, y, z = (int(v) for v in p)
        return x + self._nb[0] * (y + self._nb[1] * z)

    def __getitem__(self, p):
        flat = self.flat_index(p)
        if self.ncomp == 1:
            return BlockField(self, flat, 0)
        return TensorBlock(self, flat)

    def __iter__(self):
        for i in range(self.size()):
            yield self[i]

    def field(self, block, comp=0):
        return BlockField(self, self.flat_index(block), comp)

    # -- data movement
    def device_ptr(self, comp=0):
        p = C.c_void_p()
        _lib.check(_lib.lib().cn_grid_data(self._h, comp, C.byref(p)))
        return p.value

    def tensor(self, comp=0):
        """torch view of one component's device storage: (nblocks, block_stride)."""
        import torch
        ptr = self.device_ptr(comp)
        dt = {np.dtype(np.float32): "<f4", np.dtype(np.float64): "<f8", np.dtype(np.int32): "<i4"}[self.dtype]

        class _CAI:
            __cuda_array_interface__ = {"shape": (self.size(), self.block_stride), "typestr": dt,
                                        "data": (ptr, False), "version": 3, "strides": None}
        return torch.as_tensor(_CAI(), device="cuda")

    def upload(self, host, comp=0, stream=None):
        a = np.ascontiguousarray(host, dtype=self.dtype).reshape(-1)
        if a.size != self.comp_stride:
            raise ValueError(f"expected {self.comp_stride} elements, got {a.size}")
        _lib.check(_lib.lib().cn_grid_upload(self._h, comp, a.ctypes.data_as(C.c_void_p),
                                             a.nbytes, None if stream is None else _stream_handle(stream)))
        if stream is not None:
            self._keep = a

    def download(self, comp=0):
        a = np.empty(self.comp_stride, dtype=self.dtype)
        _lib.check(_lib.lib().cn_grid_download(self._h, comp, a.ctypes.data_as(C.c_void_p),
                                               a.nbytes, None))
        return a

    def blocks_view(self, flat_array):
        """(nblocks, nz, ny, nx) view of a component array in grid layout."""
        n = self._n
        cells = n[0] * n[1] * n[2]
        return flat_array.reshape(self.size(), self.block_stride)[:, :cells].reshape(
            self.size(), n[2], n[1], n[0])

    def copy_from(self, other, stream=None):
        """Cartesian::operator= (Grid/Cartesian.h:160-169)."""
        _lib.check(_lib.lib().cn_grid_copy(self._h, other._h, _stream_handle(stream)))

    # -- boundary conditions
    def push_boundary_bc(self, bc_factory, dir, side, comp=0):
        """Push ``bc_factory(dir, side)`` onto every block touching face (dir, side)."""
        bc = bc_factory(dir, side)
        _lib.check(_lib.lib().cn_bc_push_boundary(self._h, comp, dir, side, bc.kind, C.c_double(bc.value)))
        nb = self._nb
        for flat in range(self.size()):
            bi = (flat % nb[0], (flat // nb[0]) % nb[1], flat // (nb[0] * nb[1]))
            if (side == 0 and bi[dir] == 0) or (side == 1 and bi[dir] == nb[dir] - 1):
                self._bcs[comp].setdefault(flat, []).append(bc)

    def sync_bcs(self, stream=None):
        _lib.check(_lib.lib().cn_bc_sync(self._h, _stream_handle(stream)))

    # -- lab loading (Grid/Cartesian.h:412-427)
    def loadLab(self, field, lab, c=0, d=0):
        comp = field.comp if isinstance(field, BlockField) else int(c)
        lab.loadData(field.getState().block_index, self, comp=comp)


class FaceContainerBlock:
    """The FaceContainer of one block (Block/Field.h:1532-1670): ``[d]`` is the
    face field of direction d, a scalar ``BlockField`` or, with several
    components, a ``TensorBlock`` (``[d][c]``)."""

    def __init__(self, fgrid, flat):
        self._fg, self.flat = fgrid, flat

    def __len__(self):
        return 3

    def __getitem__(self, d):
        if not 0 <= d < 3:
            raise IndexError("face direction out of range")
        return self._fg.faces[d][self.flat]

    def getState(self):
        return self._fg.faces[0].field(self.flat, 0).getState()


class FaceCartesian:
    """Grid::Cartesian<T, Mesh, EntityType::Face, RANK>: every block holds a
    FaceContainer of three face fields (directions x, y, z) with ``ncomp``
    components each, kept as three face grids (``faces[d]``).  ``field(i, c,
    d)``, ``getIndexFunctor(c, d)`` and ``loadLab(field, lab, c, d)`` follow
    the reference's component map (block i, component c, direction d) ->
    fields[i][d][c] (Block/FieldLabLoader.h:327-364, Grid/Cartesian.h:384-427).
    Created by ``Cartesian(..., entity="face")``."""

    entity = "face"

    def __init__(self, nblocks, block_cells, begin=(0.0, 0.0, 0.0), end=(1.0, 1.0, 1.0),
                 ncomp: int = 1, dtype=np.float64):
        self.faces = tuple(Cartesian(nblocks, block_cells, begin, end, ncomp=ncomp, dtype=dtype,
                                     entity="face_" + a) for a in "xyz")
        self.ncomp = self.faces[0].ncomp
        self.dtype = self.faces[0].dtype

    def close(self):
        for f in self.faces:
            f.close()

    def size(self):
        return self.faces[0].size()

    def getSize(self):
        return self.faces[0].getSize()

    def getBlockCells(self):
        return self.faces[0].getBlockCells()

    def getBlockExtent(self, d):
        """Values per block of the face field of direction d (cells + 1 along d)."""
        return self.faces[d].getBlockExtent()

    def getCellSize(self):
        return self.faces[0].getCellSize()

    def flat_index(self, p):
        return self.faces[0].flat_index(p)

    def __getitem__(self, p):
        return FaceContainerBlock(self, self.flat_index(p))

    def __iter__(self):
        for i in range(self.size()):
            yield self[i]

    def field(self, block, comp=0, d=0):
        return self.faces[d].field(block, comp)

    def getIndexFunctor(self, c=0, d=0):
        g = self.faces[d]
        return lambda p: g.field(p, c)

    def loadLab(self, field, lab, c=0, d=0):
        """Lab of component c of the face field of direction d of the block of
        ``field`` (a FaceContainerBlock or any block field of this grid)."""
        lab.loadData(field.getState().block_index, self.faces[d], comp=int(c))

    def upload(self, host, comp=0, d=0, stream=None):
        self.faces[d].upload(host, comp, stream)

    def download(self, comp=0, d=0):
        return self.faces[d].download(comp)

    def push_boundary_bc(self, bc_factory, dir, side, comp=0, d=None):
        """BCs on the boundary blocks of the face fields of direction d (all
        three directions when d is None)."""
        for dd in (range(3) if d is None else (d,)):
            self.faces[dd].push_boundary_bc(bc_factory, dir, side, comp)

    def sync_bcs(self, stream=None):
        for f in self.faces:
            f.sync_bcs(stream)
