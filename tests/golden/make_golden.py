"""Generates the golden lab / stencil fixtures in this directory.

Runs the reference's own code (Block::FieldLab, BC::*, Grid::Cartesian and the
Laplacian / gradient benchmark loops, instantiated by oracle/ref_shim.cpp and
built into oracle/_ref/libcnref.so from the reference sources) on small,
seeded inputs and stores inputs and outputs as .npz.  The cases re-state the
set-ups of the reference's unit tests:

  fieldlab_*   test/UnitTests/Block/FieldLabTest.cpp:28-41  (16^3 iota, stencil (-2,3))
  bc_*         test/UnitTests/BC/FieldAndLab.h:31-41       (16^3 iota int, stencil (-3,4))
               BC/DirichletTest.cpp, AbsorbingTest.cpp, SymmetryTest.cpp, CommonTest.cpp
  grid_*       test/UnitTests/Grid/CartesianTest.cpp:200-318 (multi-block Cartesian)
  c1_small     test/sandbox/Benchmarks/Kernel/Laplacian/Laplacian.cpp:123-130 and
               Kernel/Divergence/nova/nova.cpp:113-126 loops

Usage:  python tests/golden/make_golden.py      (needs oracle/_ref built)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402

D, A, S, B = O.BC_DIRICHLET, O.BC_ABSORBING, O.BC_SYMMETRY, O.BC_BASE


def lab_case(name, comp, nb, n, lo, hi, tens, bcl, blocks):
    labs, defs = [], []
    for b in blocks:
        lab, w = O.lab_fill(comp, nb, n, lo, hi, tens, bcl, b, use_ref=True)
        labs.append(lab)
        defs.append(w)
    meta = dict(kind="lab", nb=list(map(int, nb)), n=list(map(int, n)), lo=list(map(int, lo)),
                hi=list(map(int, hi)), tensorial=bool(tens), blocks=list(map(int, blocks)),
                bcs={str(k): v for k, v in (bcl or {}).items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), comp=comp, labs=np.stack(labs),
                        defined=np.stack(defs), meta=json.dumps(meta))


def iota_block(n, dtype):
    nbk = int(np.prod(n))
    stride = O.block_stride(n, dtype)
    a = np.zeros(stride, dtype=dtype)
    a[:nbk] = np.arange(nbk, dtype=dtype)
    return a


def main():
    rng = np.random.default_rng(20240601)
    one = (1, 1, 1)
    # FieldLabTest: self-periodic single 16^3 block, stencil (-2,3)
    c = iota_block((16, 16, 16), np.int32)
    for t in (0, 1):
        lab_case(f"fieldlab_ghosts_t{t}", c, one, (16,) * 3, (2,) * 3, (2,) * 3, t, {}, [0])
    # BC tests: 16^3 iota int, stencil (-3,4)
    dir_all = [(0, 0, D, 10), (0, 1, D, 11), (1, 0, D, 12), (1, 1, D, 13), (2, 0, D, 14), (2, 1, D, 15)]
    lab_case("bc_dirichlet", c, one, (16,) * 3, (3,) * 3, (3,) * 3, 0, {0: dir_all}, [0])
    for d, (v0, v1) in enumerate([(101, 102), (103, 104), (105, 106)]):
        lab_case(f"bc_dirichlet_t_dir{d}", c, one, (16,) * 3, (3,) * 3, (3,) * 3, 1,
                 {0: [(d, 0, D, v0), (d, 1, D, v1)]}, [0])
    abs_all = [(d, s, A, 0) for d in range(3) for s in range(2)]
    lab_case("bc_absorbing", c, one, (16,) * 3, (3,) * 3, (3,) * 3, 0, {0: abs_all}, [0])
    for d in range(3):
        lab_case(f"bc_absorbing_t_dir{d}", c, one, (16,) * 3, (3,) * 3, (3,) * 3, 1,
                 {0: [(d, 0, A, 0), (d, 1, A, 0)]}, [0])
    sym_all = [(d, s, S, 1 if s == 0 else -1) for d in range(3) for s in range(2)]
    lab_case("bc_symmetry", c, one, (16,) * 3, (3,) * 3, (3,) * 3, 0, {0: sym_all}, [0])
    for d in range(3):
        lab_case(f"bc_symmetry_t_dir{d}", c, one, (16,) * 3, (3,) * 3, (3,) * 3, 1,
                 {0: [(d, 0, S, 1), (d, 1, S, 1)]}, [0])
    # CommonTest: zero-width stencil (0,1) leaves the lab untouched
    c4 = iota_block((4, 4, 4), np.float64)
    for k, v in ((A, 0), (D, 1.0), (S, 1)):
        lab_case(f"bc_nostencil_k{k}", c4, one, (4,) * 3, (0,) * 3, (0,) * 3, 0, {0: [(0, 0, k, v)]}, [0])

    # multi-block grids
    nb, n = (3, 2, 2), (5, 4, 3)
    nbk = int(np.prod(nb))
    comp = rng.standard_normal(nbk * O.block_stride(n, np.float64))
    lab_case("grid_periodic_f64_t1", comp, nb, n, (2, 2, 2), (2, 2, 2), 1, {}, list(range(nbk)))
    lab_case("grid_periodic_f64_t0", comp, nb, n, (1, 2, 3), (2, 1, 3), 0, {}, list(range(nbk)))

    # the mixed BC pattern of the Euler case: x periodic, y absorbing, z Dirichlet
    nb, n = (2, 3, 2), (4, 4, 4)
    nbk = int(np.prod(nb))
    comp = rng.standard_normal(nbk * O.block_stride(n, np.float64))
    bcl = {}
    for b in range(nbk):
        bi = (b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1]))
        lst = []
        if bi[1] == 0:
            lst.append((1, 0, A, 0))
        if bi[1] == nb[1] - 1:
            lst.append((1, 1, A, 0))
        if bi[2] == 0:
            lst.append((2, 0, D, 0.25))
        if bi[2] == nb[2] - 1:
            lst.append((2, 1, D, -0.5))
        bcl[b] = lst
    for t in (0, 1):
        lab_case(f"grid_mixed_f64_t{t}", comp, nb, n, (3, 3, 3), (3, 3, 3), t, bcl, list(range(nbk)))

    # float32 with symmetry signs and out-of-order / repeated BCs
    nb, n = (2, 2, 3), (6, 5, 4)
    nbk = int(np.prod(nb))
    comp = rng.standard_normal(nbk * O.block_stride(n, np.float32)).astype(np.float32)
    bcl = {}
    for b in range(nbk):
        k = int(rng.integers(0, 6))
        bcl[b] = [(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 4)),
                   float(rng.choice([-1.0, 1.0, 0.5, 2.0]))) for _ in range(k)]
    for t in (0, 1):
        lab_case(f"grid_random_f32_t{t}", comp, nb, n, (2, 1, 2), (1, 2, 2), t, bcl, list(range(nbk)))

    # C1-shaped stencils on a small grid: reference FieldLab + benchmark loops
    nb, n = (2, 2, 2), (8, 8, 8)
    nbk = int(np.prod(nb))
    stride = O.block_stride(n, np.float64)
    comp = np.zeros(nbk * stride)
    h = 1.0 / 16
    for b in range(nbk):
        bi = (b % 2, (b // 2) % 2, b // 4)
        z, y, x = np.meshgrid(*[(np.arange(8) + 8 * bi[d] + 0.5) * h for d in (2, 1, 0)], indexing="ij")
        comp[b * stride:b * stride + 512] = (np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) *
                                             np.cos(2 * np.pi * z)).ravel()
    comp += rng.uniform(-1e-3, 1e-3, size=comp.size)
    ih2 = (1.0 / (h * h),) * 3
    ih = (1.0 / h,) * 3
    _, lap, grad = O.ref_c1_sweep(comp, nb, n, ih2, ih, threads=1)
    meta = dict(kind="c1", nb=list(nb), n=list(n), h=h)
    np.savez_compressed(os.path.join(HERE, "c1_small.npz"), comp=comp, lap=lap, grad=grad,
                        meta=json.dumps(meta))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
