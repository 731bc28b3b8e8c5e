"""Helpers for GPU tests: build device grids from oracle-style descriptions and
read back labs through the C ABI."""
import ctypes as C

import numpy as np


def make_grid(cn, comp, nb, n, bcl=None, ncomp=1, dtype=None, begin=(0, 0, 0), end=(1, 1, 1), entity="cell"):
    """`n`: block cells (the mesh); node / face grids hold one more entity
    along grown dimensions in the last block."""
    dtype = np.dtype(dtype or comp.dtype)
    g = cn.Grid.Cartesian(nb, n, begin, end, ncomp=ncomp, dtype=dtype, entity=entity)
    g.upload(comp.astype(dtype), 0)
    for b, lst in (bcl or {}).items():
        for (d, s, k, v) in lst:
            C_ = {0: cn.BC.Base, 1: cn.BC.Dirichlet, 2: cn.BC.Absorbing, 3: cn.BC.Symmetry}[k]
            bc = C_(d, s) if k in (0, 2) else C_(d, s, v)
            g.field(b, 0).getBC().push_back(bc)
    return g


def lab_fill_all(cn, g, lo, hi, tens, comp=0, blocks=None, apply_bc=True):
    """Fills labs of `blocks` (default: all) twice over two sentinels; returns
    (labs[nblk, Lz, Ly, Lx], written[nblk, Lz, Ly, Lx])."""
    import torch
    from cubismnova_b200 import _lib
    n = g.getBlockExtent()
    L = [n[d] + lo[d] + hi[d] for d in range(3)]
    st = _lib.stencil_struct([-v for v in lo], [v + 1 for v in hi], tens)
    b0, cnt = (0, g.size()) if blocks is None else blocks
    tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
           np.dtype(np.int32): torch.int32}[g.dtype]
    outs = []
    for sentinel in (-777, 999):
        buf = torch.full((cnt, L[2], L[1], L[0]), sentinel, dtype=tdt, device="cuda")
        _lib.check(_lib.lib().cn_lab_fill(g.handle, comp, C.byref(st), b0, cnt, 1 if apply_bc else 0,
                                          C.c_void_p(buf.data_ptr()), None))
        torch.cuda.synchronize()
        outs.append(buf.cpu().numpy())
    a, b = outs
    written = (a.view(np.uint8).reshape(a.shape + (-1,)) == b.view(np.uint8).reshape(b.shape + (-1,))).all(-1)
    return a, written
