"""Grids split into z-slabs of block layers, one per rank, with the exchange
of ghost slabs between neighbouring slabs.

The reference's multi-process form keeps blocks on MPI ranks and fills the
labs across rank boundaries through the legacy synchroniser's halo messages
(test/sandbox/Benchmarks/CubismLegacy/include/Cubism/SynchronizerMPI.h:826-876:
pack the boundary cells each neighbour needs, exchange, unpack into the
ghost region).  Here a rank holds its slab of block layers plus one ghost
block layer below and one above in an ordinary ``Grid.Cartesian`` of the same
cell size, so that every kernel (lab fill, stencils, the Euler stages) runs on
the slab unchanged: before a stencil the ``depth`` cell planes next to each
slab face are packed on the device (``cn_grid_to_aos``), exchanged, and
unpacked into the neighbours' ghost layers (``cn_grid_from_aos``).  Only the
owned layers' results are meaningful; the ghost layers are scratch.

Slabs form a ring along z (periodic z); with BCs on the global z faces the
slabs holding them carry those BCs on their owned boundary layers, which
makes their labs skip the ghost layer exactly as the global grid's labs skip
the periodic neighbour.  Transports: ``exchange_local`` between slabs held by
one process (a device copy per message), ``exchange`` over
``torch.distributed`` point-to-point messages (NCCL on GPUs; gloo for the
host-side tests).
"""
from __future__ import annotations

import numpy as np

from . import euler as _euler
from .grid import Cartesian


def split_layers(nbz: int, world: int):
    """Block layers [z0, z1) of every rank: contiguous, sizes differing by at
    most one, the larger ones first."""
    if world < 1 or nbz < world:
        raise ValueError(f"{nbz} block layers can not be split over {world} ranks")
    base, extra = divmod(nbz, world)
    out, z = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((z, z + k))
        z += k
    return out


class ZSlab:
    """Rank ``rank`` of ``world``: block layers [z0, z1) of a global grid of
    ``nb`` blocks of ``n`` cells over [begin, end); its local grid has
    (nb[0], nb[1], z1 - z0 + 2) blocks, local layer 0 and the last one being
    the ghost layers."""

    def __init__(self, nb, n, rank: int, world: int, begin=(0.0, 0.0, 0.0), end=(1.0, 1.0, 1.0)):
        self.nb_global = tuple(int(v) for v in nb)
        self.n = tuple(int(v) for v in n)
        self.rank, self.world = int(rank), int(world)
        self.z0, self.z1 = split_layers(self.nb_global[2], self.world)[self.rank]
        self.own = self.z1 - self.z0
        self.nb = (self.nb_global[0], self.nb_global[1], self.own + 2)
        self.begin_global, self.end_global = tuple(begin), tuple(end)
        hz = (end[2] - begin[2]) / (self.nb_global[2] * self.n[2])
        self.begin = (begin[0], begin[1], begin[2] + (self.z0 - 1) * self.n[2] * hz)
        self.end = (end[0], end[1], begin[2] + (self.z1 + 1) * self.n[2] * hz)
        self.down = (self.rank - 1) % self.world  # the slab below (ring)
        self.up = (self.rank + 1) % self.world

    def grid(self, ncomp: int = 1, dtype=np.float64) -> Cartesian:
        """The local grid (owned layers and the two ghost layers)."""
        return Cartesian(self.nb, self.n, self.begin, self.end, ncomp=ncomp, dtype=dtype)

    def global_block(self, local_flat: int) -> int:
        """Global flat index of a local block (-1 for a ghost-layer block)."""
        nbx, nby = self.nb[0], self.nb[1]
        bz = local_flat // (nbx * nby)
        if bz == 0 or bz == self.own + 1:
            return -1
        return local_flat + (self.z0 - 1) * nbx * nby

    def owned_local_blocks(self):
        """Local flat indices of the owned blocks, in global block order."""
        nxy = self.nb[0] * self.nb[1]
        return list(range(nxy, (self.own + 1) * nxy))

    def push_boundary_bc(self, grid: Cartesian, bc_factory, dir: int, side: int, comp: int = 0):
        """The global grid's push_boundary_bc on this slab: x and y faces on
        every owned block touching them; a z face only on the slab holding it
        (its first or last owned layer).  Ghost layers get none."""
        nb = self.nb
        for flat in self.owned_local_blocks():
            bi = (flat % nb[0], (flat // nb[0]) % nb[1], flat // (nb[0] * nb[1]))
            if dir < 2:
                on = bi[dir] == (0 if side == 0 else nb[dir] - 1)
            else:
                on = (side == 0 and self.z0 == 0 and bi[2] == 1) or \
                     (side == 1 and self.z1 == self.nb_global[2] and bi[2] == self.own)
            if on:
                grid.field(flat, comp).getBC().push_back(bc_factory(dir, side))

    # -- the ghost slabs: local cell planes along z (global entity indices of the local grid)
    def _span(self, kind: str, depth: int):
        nz = self.n[2]
        top = (self.own + 1) * nz
        z = {"send_low": (nz, nz + depth), "send_high": (top - depth, top),
             "recv_low": (nz - depth, nz), "recv_high": (top, top + depth)}[kind]
        ext = (self.nb[0] * self.n[0], self.nb[1] * self.n[1])
        return (0, 0, z[0]), (ext[0], ext[1], z[1])

    def pack(self, grid: Cartesian, side: int, depth: int, comps=None, stream=None):
        """The ``depth`` owned cell planes next to face ``side`` (0 low, 1
        high) as a device buffer (z, y, x, components)."""
        from . import io as IO
        if depth < 1 or depth > self.n[2]:
            raise ValueError("ghost depth must be in [1, block cells along z]")
        return IO.Field2AOS(grid, self._span("send_low" if side == 0 else "send_high", depth), comps=comps,
                            stream=stream)

    def unpack(self, grid: Cartesian, side: int, depth: int, buf, comps=None, stream=None):
        """A neighbour's packed planes into the ghost layer on side ``side``."""
        from . import io as IO
        IO.AOS2Field(buf, grid, self._span("recv_low" if side == 0 else "recv_high", depth), comps=comps,
                     stream=stream)


def exchange_local(slabs, grids, depth: int, comps=None, stream=None):
    """Ghost exchange between the slabs of one process (``slabs[r]`` the
    slab of rank r of the ring, ``grids[r]`` its local grid)."""
    world = len(slabs)
    lows = [slabs[r].pack(grids[r], 0, depth, comps, stream) for r in range(world)]
    highs = [slabs[r].pack(grids[r], 1, depth, comps, stream) for r in range(world)]
    for r in range(world):
        s = slabs[r]
        s.unpack(grids[r], 1, depth, lows[s.up], comps, stream)    # above me: the next slab's lowest planes
        s.unpack(grids[r], 0, depth, highs[s.down], comps, stream)  # below me: the previous slab's top planes


def exchange_messages(slab: ZSlab, low, high, group=None):
    """Point-to-point part of ``exchange`` on host or device tensors: sends
    ``low`` (this slab's lowest planes) to the slab below and ``high`` to the
    one above; returns (from_up, from_down), the buffers for the high and the
    low ghost layer.  Messages are posted in one fixed order on every rank
    (send low, send high, receive from above, receive from below), so that
    with two ranks, where both neighbours are the same rank, the pairs match
    in order."""
    import torch
    import torch.distributed as dist
    if slab.world == 1:
        return low.clone(), high.clone()
    from_up, from_down = torch.empty_like(low), torch.empty_like(high)
    ranks = (lambda r: dist.get_global_rank(group, r)) if group is not None else (lambda r: r)
    ops = [dist.P2POp(dist.isend, low.contiguous(), ranks(slab.down), group, tag=0),
           dist.P2POp(dist.isend, high.contiguous(), ranks(slab.up), group, tag=1),
           dist.P2POp(dist.irecv, from_up, ranks(slab.up), group, tag=0),
           dist.P2POp(dist.irecv, from_down, ranks(slab.down), group, tag=1)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    return from_up, from_down


def exchange(slab: ZSlab, grid: Cartesian, depth: int, comps=None, group=None, stream=None):
    """Ghost exchange of one rank over torch.distributed: pack on the
    device, exchange the two messages with the neighbouring slabs, unpack."""
    import torch
    low = slab.pack(grid, 0, depth, comps, stream)
    high = slab.pack(grid, 1, depth, comps, stream)
    if stream is not None:
        stream.synchronize()
    else:
        torch.cuda.synchronize()
    from_up, from_down = exchange_messages(slab, low, high, group)
    slab.unpack(grid, 1, depth, from_up, comps, stream)
    slab.unpack(grid, 0, depth, from_down, comps, stream)


def rk3_step(U: Cartesian, w1: Cartesian, w2: Cartesian, dt: float, exchange_fn, gamma: float = _euler.GAMMA,
             stream=None):
    """One SSP-RK3 step of the Euler equations on a slab: before each stage
    the stage's input gets fresh ghost layers (``exchange_fn(grid)``, 3 cell
    planes: the stencil (-3, 4)); U holds the BCs (it is the BC source of all
    three stages)."""
    exchange_fn(U)
    _euler.rk3_stage(U, U, None, w1, 1, dt, gamma, stream=stream)
    exchange_fn(w1)
    _euler.rk3_stage(U, w1, U, w2, 2, dt, gamma, stream=stream)
    exchange_fn(w2)
    _euler.rk3_stage(U, w2, U, U, 3, dt, gamma, stream=stream)


def rk3_step_local(slabs, Us, w1s, w2s, dt: float, gamma: float = _euler.GAMMA, stream=None):
    """``rk3_step`` for the slabs of one process together: each stage's
    inputs of all slabs are exchanged (``exchange_local``), then the stage
    runs on every slab."""
    depth = 3
    exchange_local(slabs, Us, depth, stream=stream)
    for U, w1 in zip(Us, w1s):
        _euler.rk3_stage(U, U, None, w1, 1, dt, gamma, stream=stream)
    exchange_local(slabs, w1s, depth, stream=stream)
    for U, w1, w2 in zip(Us, w1s, w2s):
        _euler.rk3_stage(U, w1, U, w2, 2, dt, gamma, stream=stream)
    exchange_local(slabs, w2s, depth, stream=stream)
    for U, w2 in zip(Us, w2s):
        _euler.rk3_stage(U, w2, U, U, 3, dt, gamma, stream=stream)
