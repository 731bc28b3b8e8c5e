"""Array-of-structures file buffers of a grid: CPU restatement.

TEST INFRASTRUCTURE ONLY (oracle of cn_grid_to_aos / cn_grid_from_aos).

Restates the block loop of IO::CartesianWriteHDF / CartesianReadHDF
(IO/CartesianHDF.h:76-80, 182-186) over Field2AOS / AOS2Field
(IO/FieldAOS.h:37-77 scalar, :79-124 tensor, :136-149 face container): for
every block field, the intersection of the file index range r with the
block's global index range (Core/Range.h:216-228; an empty overlap in any
dimension copies nothing) is copied point by point,
    buf[c + ncomp * r.getFlatIndexFromGlobal(p)] = field_c[p]   (write)
    field_c[p] = buf[c + ncomp * r.getFlatIndexFromGlobal(p)]   (read)
converting between the grid's and the file's type as C++ assignment does
(numpy astype: double -> float rounds to nearest even).  Blocks hold cells,
or cells + 1 nodes / faces along grown dimensions in the last block
(Grid/BlockFieldAssembler.h:124-135); block data is dense with the block's
own extent, blocks `block_stride` elements apart.  Pinned against the
reference's own Field2AOS / AOS2Field through oracle/_ref (ref_field_aos_*).
"""
import numpy as np

ENTITY_GROW = {0: (0, 0, 0), 1: (1, 1, 1), 2: (1, 0, 0), 3: (0, 1, 0), 4: (0, 0, 1)}


def _blocks(nb, cells, entity):
    grow = ENTITY_GROW[entity]
    for bz in range(nb[2]):
        for by in range(nb[1]):
            for bx in range(nb[0]):
                bi = (bx, by, bz)
                ext = tuple(cells[d] + (1 if grow[d] and bi[d] == nb[d] - 1 else 0) for d in range(3))
                beg = tuple(bi[d] * cells[d] for d in range(3))
                yield bx + nb[0] * (by + nb[1] * bz), beg, ext


def _overlap(beg, ext, sb, se):
    lo = [max(beg[d], sb[d]) for d in range(3)]
    hi = [min(beg[d] + ext[d], sb[d] + se[d]) for d in range(3)]
    if any(hi[d] <= lo[d] for d in range(3)):
        return None
    return lo, hi


def grid_to_aos(comps, nb, cells, entity, block_stride, span_begin, span_end, out):
    """comps: list of ncomp component arrays (grid layout); out: flat buffer of
    span volume * ncomp values of the file type, written where the span meets
    the grid (other values are left as they are).  Returns out."""
    sb, se = list(span_begin), [span_end[d] - span_begin[d] for d in range(3)]
    nc = len(comps)
    o4 = out.reshape(se[2], se[1], se[0], nc)
    for flat, beg, ext in _blocks(nb, cells, entity):
        ov = _overlap(beg, ext, sb, se)
        if ov is None:
            continue
        lo, hi = ov
        for c in range(nc):
            blk = comps[c][flat * block_stride: flat * block_stride + ext[0] * ext[1] * ext[2]]
            blk = blk.reshape(ext[2], ext[1], ext[0])
            sub = blk[lo[2] - beg[2]:hi[2] - beg[2], lo[1] - beg[1]:hi[1] - beg[1], lo[0] - beg[0]:hi[0] - beg[0]]
            o4[lo[2] - sb[2]:hi[2] - sb[2], lo[1] - sb[1]:hi[1] - sb[1], lo[0] - sb[0]:hi[0] - sb[0], c] = \
                sub.astype(out.dtype)
    return out


def aos_to_grid(buf, comps, nb, cells, entity, block_stride, span_begin, span_end):
    """Reads buf (span volume * ncomp file values) into copies of comps where
    the span meets the grid; returns the new component arrays."""
    sb, se = list(span_begin), [span_end[d] - span_begin[d] for d in range(3)]
    nc = len(comps)
    out = [np.array(c, copy=True) for c in comps]
    b4 = buf.reshape(se[2], se[1], se[0], nc)
    for flat, beg, ext in _blocks(nb, cells, entity):
        ov = _overlap(beg, ext, sb, se)
        if ov is None:
            continue
        lo, hi = ov
        for c in range(nc):
            blk = out[c][flat * block_stride: flat * block_stride + ext[0] * ext[1] * ext[2]]
            blk = blk.reshape(ext[2], ext[1], ext[0])
            blk[lo[2] - beg[2]:hi[2] - beg[2], lo[1] - beg[1]:hi[1] - beg[1], lo[0] - beg[0]:hi[0] - beg[0]] = \
                b4[lo[2] - sb[2]:hi[2] - sb[2], lo[1] - sb[1]:hi[1] - sb[1], lo[0] - sb[0]:hi[0] - sb[0], c] \
                .astype(out[c].dtype)
    return out
