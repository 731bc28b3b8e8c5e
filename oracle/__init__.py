"""CPU oracle for the lab-fill / stencil hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
package ``cubismnova_b200`` never imports it.

Two libraries sit behind it:

* ``liboracle.so`` -- the plain-C restatement (``cn_oracle.c`` and friends),
  built from this directory by ``make``;
* ``_ref/libcnref.so`` -- the reference's own header-only C++ code
  (``Block/FieldLab.h``, ``BC/*.h``, ``Grid/Cartesian.h``) instantiated by
  ``ref_shim.cpp``; present only where it was built from the reference
  sources.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

BC_BASE, BC_DIRICHLET, BC_ABSORBING, BC_SYMMETRY = 0, 1, 2, 3


class OrBC(C.Structure):
    _fields_ = [("dir", C.c_int32), ("side", C.c_int32), ("kind", C.c_int32),
                ("pad", C.c_int32), ("value", C.c_double)]


class OrGeom(C.Structure):
    _fields_ = [("nb", C.c_int32 * 3), ("n", C.c_int32 * 3), ("lo", C.c_int32 * 3),
                ("hi", C.c_int32 * 3), ("tensorial", C.c_int32),
                ("block_stride", C.c_int64), ("grow", C.c_int32 * 3)]


_lib = None
_ref = None


def build(quiet: bool = True) -> None:
    """Run ``make`` in this directory (oracle + reference shim if possible)."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libcnref.so"))


def ref():
    global _ref
    if _ref is None:
        path = os.path.join(_HERE, "_ref", "libcnref.so")
        if not os.path.exists(path):
            raise FileNotFoundError("reference shim not built: " + path)
        _ref = C.CDLL(path)
        _ref.ref_c1_sweep_f64.restype = C.c_double
    return _ref


def block_stride(n, dtype) -> int:
    """Elements between blocks: cells*sizeof rounded up to 32 B
    (Grid/Cartesian.h:490-513)."""
    itemsize = np.dtype(dtype).itemsize
    cells = int(n[0]) * int(n[1]) * int(n[2])
    nbytes = (cells * itemsize + 31) // 32 * 32
    return nbytes // itemsize


ENTITY_GROW = {0: (0, 0, 0), 1: (1, 1, 1), 2: (1, 0, 0), 3: (0, 1, 0), 4: (0, 0, 1)}


def make_geom(nb, n, lo, hi, tensorial, stride, entity=0) -> OrGeom:
    g = OrGeom()
    for d in range(3):
        g.nb[d], g.n[d], g.lo[d], g.hi[d] = int(nb[d]), int(n[d]), int(lo[d]), int(hi[d])
        g.grow[d] = ENTITY_GROW[entity][d]
    g.tensorial = 1 if tensorial else 0
    g.block_stride = int(stride)
    return g


def bc_arrays(nblocks: int, bclists):
    """CSR (offsets, entries) from a dict block -> list of (dir, side, kind, value)."""
    off = np.zeros(nblocks + 1, dtype=np.int32)
    ents = []
    for b in range(nblocks):
        lst = bclists.get(b, []) if bclists else []
        off[b + 1] = off[b] + len(lst)
        for (d, s, k, v) in lst:
            e = OrBC()
            e.dir, e.side, e.kind, e.value = int(d), int(s), int(k), float(v)
            ents.append(e)
    arr = (OrBC * max(1, len(ents)))(*ents) if ents else (OrBC * 1)()
    return off, arr


_SUFFIX = {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32",
           np.dtype(np.int32): "i32"}


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def entity_stride(cells, entity, dtype) -> int:
    """Block stride of a node (entity 1) or face (2..4) grid: (cells + 1)^3
    slots rounded to 32 bytes (Grid/Cartesian.h:490-513); cells for entity 0."""
    ext = [int(c) + (0 if entity == 0 else 1) for c in cells]
    return block_stride(ext, dtype)


def lab_fill(comp, nb, n, lo, hi, tensorial, bclists, block, use_ref=False,
             lab_init=None, stride=None, entity=0):
    """Lab of one block: returns (lab[Lz,Ly,Lx], defined[Lz,Ly,Lx] bool).
    `n` is the largest block extent (cells, or cells + 1 for nodes and along
    a face direction, where only the last block along that dimension has it);
    `stride` the block stride (default: the cell layout of `n`); `entity`
    (cn_entity numbering) selects node / face fields."""
    comp = np.ascontiguousarray(comp)
    sfx = _SUFFIX[comp.dtype]
    stride = block_stride(n, comp.dtype) if stride is None else int(stride)
    g = make_geom(nb, n, lo, hi, tensorial, stride, entity)
    nblocks = int(np.prod(nb))
    off, ents = bc_arrays(nblocks, bclists)
    L = [int(n[d]) + int(lo[d]) + int(hi[d]) for d in range(3)]
    lab = np.zeros((L[2], L[1], L[0]), dtype=comp.dtype) if lab_init is None \
        else np.array(lab_init, dtype=comp.dtype, copy=True)
    w = np.zeros((L[2], L[1], L[0]), dtype=np.uint8)
    if use_ref and entity != 0:
        if comp.dtype != np.float64:
            raise ValueError("node/face reference labs are built for float64")
        rc = ref().ref_lab_fill_entity_f64(C.byref(g), C.c_int(entity), _ptr(comp), _ptr(off), ents, C.c_int(block),
                                           _ptr(lab), _ptr(w))
    else:
        f = getattr(ref() if use_ref else lib(), ("ref_" if use_ref else "or_") + "lab_fill_" + sfx)
        rc = f(C.byref(g), _ptr(comp), _ptr(off), ents, C.c_int(block), _ptr(lab), _ptr(w))
    if rc != 0:
        raise ValueError("lab fill rejected the geometry")
    return lab, w.astype(bool)


def laplacian_f64(comp, nb, n, bclists, ih2):
    comp = np.ascontiguousarray(comp, dtype=np.float64)
    stride = block_stride(n, np.float64)
    g = make_geom(nb, n, (1, 1, 1), (1, 1, 1), False, stride)
    off, ents = bc_arrays(int(np.prod(nb)), bclists)
    out = np.zeros_like(comp)
    ih2a = (C.c_double * 3)(*[float(v) for v in ih2])
    rc = lib().or_laplacian_f64(C.byref(g), _ptr(comp), _ptr(off), ents, ih2a, _ptr(out))
    if rc:
        raise ValueError("or_laplacian_f64 failed")
    return out


def gradient_f64(comp, nb, n, bclists, ih):
    comp = np.ascontiguousarray(comp, dtype=np.float64)
    stride = block_stride(n, np.float64)
    g = make_geom(nb, n, (1, 1, 1), (1, 1, 1), False, stride)
    off, ents = bc_arrays(int(np.prod(nb)), bclists)
    out = np.zeros((3,) + comp.shape, dtype=np.float64)
    iha = (C.c_double * 3)(*[float(v) for v in ih])
    rc = lib().or_gradient_f64(C.byref(g), _ptr(comp), _ptr(off), ents, iha, _ptr(out),
                               C.c_int64(comp.size))
    if rc:
        raise ValueError("or_gradient_f64 failed")
    return out


def ref_c1_sweep(comp, nb, n, ih2, ih, threads=0, nblocks=0, reps=1,
                 want_lap=True, want_grad=True):
    """Reference FieldLab + Laplacian/gradient loops with OpenMP; returns
    (seconds per sweep, lap, grad)."""
    comp = np.ascontiguousarray(comp, dtype=np.float64)
    stride = block_stride(n, np.float64)
    lap = np.zeros_like(comp) if want_lap else None
    grad = np.zeros((3,) + comp.shape, dtype=np.float64) if want_grad else None
    nba = (C.c_int * 3)(*[int(v) for v in nb])
    na = (C.c_int * 3)(*[int(v) for v in n])
    t = ref().ref_c1_sweep_f64(
        nba, na, _ptr(comp), C.c_int64(stride),
        _ptr(lap) if lap is not None else None,
        _ptr(grad) if grad is not None else None, C.c_int64(comp.size),
        (C.c_double * 3)(*ih2), (C.c_double * 3)(*ih),
        C.c_int(threads if threads > 0 else (os.cpu_count() or 1)),
        C.c_int(nblocks), C.c_int(reps))
    return t, lap, grad


def euler_stage(Us, Un, nb, n, bclists, stage, dt, gamma, h, threads=0):
    """Euler RHS (stage 0) or SSP-RK3 stage on (5, comp_stride) arrays.
    bclists: list of 5 dicts block -> [(dir, side, kind, value)]."""
    Us = np.ascontiguousarray(Us)
    dt_ = Us.dtype
    sfx = {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32"}[dt_]
    stride = block_stride(n, dt_)
    g = make_geom(nb, n, (3, 3, 3), (3, 3, 3), False, stride)
    nblocks = int(np.prod(nb))
    offs, ents = [], []
    for c in range(5):
        o, e = bc_arrays(nblocks, (bclists[c] if bclists else {}))
        offs.append(o)
        ents.append(e)
    off_ptrs = (C.c_void_p * 5)(*[o.ctypes.data for o in offs])
    ent_ptrs = (C.c_void_p * 5)(*[C.addressof(e) for e in ents])
    out = np.array(Un, copy=True) if (Un is not None and stage == 3) else np.zeros_like(Us)
    Unp = _ptr(np.ascontiguousarray(Un)) if Un is not None else None
    f = getattr(lib(), "or_euler_stage_" + sfx)
    rc = f(C.byref(g), _ptr(Us), Unp, _ptr(out), C.c_int64(Us.shape[-1]), off_ptrs, ent_ptrs,
           C.c_int(stage), C.c_double(dt), C.c_double(gamma), (C.c_double * 3)(*h),
           C.c_int(threads if threads > 0 else (os.cpu_count() or 1)))
    if rc:
        raise ValueError("or_euler_stage failed")
    return out


def euler_rk3_step(U, nb, n, bclists, dt, gamma, h, threads=0):
    U1 = euler_stage(U, None, nb, n, bclists, 1, dt, gamma, h, threads)
    U2 = euler_stage(U1, U, nb, n, bclists, 2, dt, gamma, h, threads)
    return euler_stage(U2, U, nb, n, bclists, 3, dt, gamma, h, threads)


def ref_lab_sweep(comps, nb, n, bclists, lo, hi, threads=0, reps=1):
    """The labs of every block of each component of ``comps`` (rows in the
    grid layout) loaded by the reference FieldLab (oracle/_ref), stencil
    (-lo, hi+1) non-tensorial; returns the best seconds per sweep."""
    comps = np.ascontiguousarray(comps, dtype=np.float64)
    ncomp = comps.shape[0]
    stride = block_stride(n, np.float64)
    nblocks = int(np.prod(nb))
    offs, ents = [], []
    for c in range(ncomp):
        o, e = bc_arrays(nblocks, (bclists[c] if bclists else {}))
        offs.append(o)
        ents.append(e)
    off_ptrs = (C.c_void_p * ncomp)(*[o.ctypes.data for o in offs])
    ent_ptrs = (C.c_void_p * ncomp)(*[C.addressof(e) for e in ents])
    f = ref().ref_lab_sweep_f64
    f.restype = C.c_double
    return f((C.c_int * 3)(*nb), (C.c_int * 3)(*n), _ptr(comps), C.c_int64(stride), C.c_int64(comps.shape[-1]),
             off_ptrs, ent_ptrs, C.c_int(ncomp), C.c_int(lo), C.c_int(hi),
             C.c_int(threads if threads > 0 else (os.cpu_count() or 1)), C.c_int(reps))


def ref_euler_stage(Us, Un, nb, n, bclists, stage, dt, gamma, h, threads=0, blocks=None, reps=1):
    """The Euler stage with labs loaded by the reference FieldLab (oracle/_ref).
    Returns (seconds for the sampled blocks, out)."""
    Us = np.ascontiguousarray(Us, dtype=np.float64)
    stride = block_stride(n, np.float64)
    nblocks = int(np.prod(nb))
    offs, ents = [], []
    for c in range(5):
        o, e = bc_arrays(nblocks, (bclists[c] if bclists else {}))
        offs.append(o)
        ents.append(e)
    off_ptrs = (C.c_void_p * 5)(*[o.ctypes.data for o in offs])
    ent_ptrs = (C.c_void_p * 5)(*[C.addressof(e) for e in ents])
    out = np.array(Un, copy=True) if (Un is not None and stage == 3) else np.zeros_like(Us)
    b0, cnt = (0, nblocks) if blocks is None else blocks
    f = ref().ref_euler_stage_f64
    f.restype = C.c_double
    t = f((C.c_int * 3)(*nb), (C.c_int * 3)(*n), _ptr(Us),
          _ptr(np.ascontiguousarray(Un)) if Un is not None else None, _ptr(out),
          C.c_int64(stride), C.c_int64(Us.shape[-1]), off_ptrs, ent_ptrs, C.c_int(stage),
          C.c_double(dt), C.c_double(gamma), (C.c_double * 3)(*h),
          C.c_int(threads if threads > 0 else (os.cpu_count() or 1)), C.c_int(b0), C.c_int(cnt),
          C.c_int(reps))
    return t, out


# ------------------------------------------------------------------ IO (AoS)
def ref_field_aos(data, nb, cells, entity, block_stride, span_begin, span_end, file_dtype, buf, to_aos=True,
                  threads=1, reps=1):
    """The reference's Field2AOS (to_aos) or AOS2Field block loop
    (IO/CartesianHDF.h:76-80, 182-186) on a reference grid built from
    `data` ((ncomp, comp_stride) array, grid layout; ncomp 1, or 3 for
    cells).  Writes `buf` (to_aos) or returns the grid data after reading it.
    Returns (best seconds per pass, data)."""
    data = np.array(data, copy=True, order="C")
    sfx = {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32"}[data.dtype]
    f = getattr(ref(), "ref_field_aos_" + sfx)
    f.restype = C.c_double
    fd = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}[np.dtype(file_dtype)]
    se = [span_end[d] - span_begin[d] for d in range(3)]
    assert buf.dtype == np.dtype(file_dtype) and buf.size == int(np.prod(se)) * data.shape[0]
    t = f((C.c_int * 3)(*nb), (C.c_int * 3)(*cells), C.c_int(entity), C.c_int(data.shape[0]), _ptr(data),
          C.c_int64(data.shape[1]), C.c_int64(block_stride), (C.c_int * 3)(*span_begin), (C.c_int * 3)(*se),
          C.c_int(fd), _ptr(buf), C.c_int(1 if to_aos else 0), C.c_int(threads), C.c_int(reps))
    if t < 0:
        raise ValueError("ref_field_aos: unsupported entity / component count")
    return t, data


# ---------------------------------------------------------------- multigrid
def _i3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def _f32p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def mg_jacobi(pin, k, f, nb, n, omega, ih2):
    out = np.zeros_like(f)
    s = block_stride(n, np.float32)
    lib().or_mg_jacobi(_i3(nb), _i3(n), C.c_int64(s), _f32p(pin), _f32p(k), _f32p(f),
                       C.c_float(omega), C.c_float(ih2), _f32p(out))
    return out


def mg_resid_restrict(p, k, f, nb, n, ih2):
    nc = [v // 2 for v in n]
    cs = block_stride(nc, np.float32)
    out = np.zeros(int(np.prod(nb)) * cs, dtype=np.float32)
    lib().or_mg_resid_restrict(_i3(nb), _i3(n), C.c_int64(block_stride(n, np.float32)), _f32p(p), _f32p(k),
                               _f32p(f), C.c_float(ih2), C.c_int64(cs), _f32p(out))
    return out


def mg_restrict_mean(kf, nb, n):
    nc = [v // 2 for v in n]
    cs = block_stride(nc, np.float32)
    out = np.zeros(int(np.prod(nb)) * cs, dtype=np.float32)
    lib().or_mg_restrict_mean(_i3(nb), _i3(n), C.c_int64(block_stride(n, np.float32)), _f32p(kf),
                              C.c_int64(cs), _f32p(out))
    return out


def mg_prolong(p, e, nb, n):
    out = np.array(p, dtype=np.float32, copy=True)
    nc = [v // 2 for v in n]
    lib().or_mg_prolong(_i3(nb), _i3(n), C.c_int64(block_stride(n, np.float32)), _f32p(out),
                        C.c_int64(block_stride(nc, np.float32)), _f32p(e))
    return out


def mg_resid64(p64, k, f, nb, n, ih2):
    r32 = np.zeros_like(f)
    rr, ff = C.c_double(), C.c_double()
    lib().or_mg_resid64(_i3(nb), _i3(n), C.c_int64(block_stride(n, np.float64)), _ptr(p64),
                        C.c_int64(block_stride(n, np.float32)), _f32p(k), _f32p(f), C.c_double(ih2),
                        _f32p(r32), C.byref(rr), C.byref(ff))
    return r32, rr.value, ff.value


def mg_coarse_cg(f, k, nb, n, ih2, max_iter=10000, rtol=1e-13):
    p = np.zeros_like(f)
    it = lib().or_mg_coarse_cg(_i3(nb), _i3(n), C.c_int64(block_stride(n, np.float32)), _f32p(f), _f32p(k),
                               C.c_double(ih2), C.c_int(max_iter), C.c_double(rtol), _f32p(p))
    return p, it


def _blocks(a, nb, n, dtype):
    """(nblocks, cells) view of a block-strided component."""
    nblk, cells = int(np.prod(nb)), int(np.prod(n))
    return a.reshape(nblk, block_stride(n, dtype))[:, :cells]


def mg_solve(k, f, nb, n, h, nu1=2, nu2=2, omega=0.8, rtol=1e-8, max_cycles=100):
    """The device solver's algorithm on the CPU: FP32 V-cycles (levels halve
    the block cells while even; weighted Jacobi, nu1 from a zero guess / nu2;
    fused residual restriction; trilinear prolongation; CG on the coarsest
    level) inside an FP64 defect correction p64 += V(r32), from p64 = 0 until
    ||r|| <= rtol ||f||.  Returns (p64, cycles, relres)."""
    ks, ns = [k], [list(n)]
    while all(v % 2 == 0 for v in ns[-1]):
        ks.append(mg_restrict_mean(ks[-1], nb, ns[-1]))
        ns.append([v // 2 for v in ns[-1]])
    ih2 = [1.0 / (h * 2 ** l) ** 2 for l in range(len(ns))]

    def vcycle(l, fl):
        if l == len(ns) - 1:
            return mg_coarse_cg(fl, ks[l], nb, ns[l], ih2[l])[0]
        p = None
        for _ in range(nu1):
            p = mg_jacobi(p, ks[l], fl, nb, ns[l], omega, ih2[l])
        if p is None:
            p = np.zeros_like(fl)
        fc = mg_resid_restrict(p, ks[l], fl, nb, ns[l], ih2[l])
        p = mg_prolong(p, vcycle(l + 1, fc), nb, ns[l])
        for _ in range(nu2):
            p = mg_jacobi(p, ks[l], fl, nb, ns[l], omega, ih2[l])
        return p

    p64 = np.zeros(int(np.prod(nb)) * block_stride(n, np.float64))
    r32, rr, ff = mg_resid64(p64, k, f, nb, n, ih2[0])
    fn = np.sqrt(ff)
    rel = np.sqrt(rr) / fn if fn > 0 else 0.0
    cycles = 0
    while cycles < max_cycles and rel > rtol:
        e = vcycle(0, r32)
        _blocks(p64, nb, n, np.float64)[:] += _blocks(e, nb, n, np.float32).astype(np.float64)
        r32, rr, _ = mg_resid64(p64, k, f, nb, n, ih2[0])
        rel = np.sqrt(rr) / fn
        cycles += 1
    return p64, cycles, rel


# ---------------------------------------------------------------------- AMR
AMR_BLOCK = np.dtype([("level", "<i4"), ("n", "<i4"), ("ox", "<i4"), ("oy", "<i4"), ("oz", "<i4"),
                      ("pad", "<i4"), ("off", "<i8"), ("ih", "<f8")])


def _extents(L1):
    """Box extents (Lx, Ly, Lz) in level-1 cells from one extent or three."""
    return (C.c_int * 3)(*[int(e) for e in np.broadcast_to(np.asarray(L1), (3,))])


def amr_blocks(levels, cells, origins, L1):
    """Oracle block table (offsets: blocks contiguous in block order); L1 is
    the box extent in level-1 cells, one value (cube) or (Lx, Ly, Lz); cells
    are cubic with h = cell size / Lx."""
    nb = len(levels)
    blk = np.zeros(nb, dtype=AMR_BLOCK)
    off = 0
    lx = int(np.broadcast_to(np.asarray(L1), (3,))[0])
    for b in range(nb):
        cs = 2 if levels[b] == 0 else 1
        blk[b] = (levels[b], cells[b], origins[b][0], origins[b][1], origins[b][2], 0, off, lx / cs)
        off += cells[b] ** 3
    return blk, off


def amr_lab(comp, blk, L1, b, g):
    n = int(blk[b]["n"])
    E = n + 2 * g
    lab = np.zeros((E, E, E))
    w = np.zeros((E, E, E), dtype=np.uint8)
    rc = lib().or_amr_lab_f64(blk.ctypes.data_as(C.c_void_p), C.c_int(len(blk)), _extents(L1),
                              _ptr(np.ascontiguousarray(comp, dtype=np.float64)), C.c_int(b), C.c_int(g),
                              _ptr(lab), _ptr(w))
    if rc:
        raise ValueError("or_amr_lab_f64 failed")
    return lab, w.astype(bool)


def amr_stage(Us, Un, blk, L1, stage, dt, gamma):
    Us = np.ascontiguousarray(Us, dtype=np.float64)
    out = np.array(Un, copy=True) if (Un is not None and stage == 3) else np.zeros_like(Us)
    rc = lib().or_amr_stage_f64(blk.ctypes.data_as(C.c_void_p), C.c_int(len(blk)), _extents(L1), _ptr(Us),
                                _ptr(np.ascontiguousarray(Un)) if Un is not None else None, _ptr(out),
                                C.c_int64(Us.shape[-1]), C.c_int(stage), C.c_double(dt), C.c_double(gamma))
    if rc:
        raise ValueError("or_amr_stage_f64 failed")
    return out
