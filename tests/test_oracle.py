"""The CPU oracle pinned against the reference (CPU only, no GPU).

* against the golden fixtures produced by the reference's own FieldLab / BC /
  Cartesian code (tests/golden/make_golden.py);
* against the reference built here (oracle/_ref) on randomised geometries,
  stencils and BC vectors, when that build is present;
* the assertions of the reference's unit tests, re-expressed on oracle labs.
"""
import numpy as np
import pytest

import labchecks as LC
from golden_io import c1_small, lab_cases

CASES = lab_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_golden(oracle_lib, case):
    O = oracle_lib
    for i, b in enumerate(case["blocks"]):
        lab, w = O.lab_fill(case["comp"], case["nb"], case["n"], case["lo"], case["hi"],
                            case["tensorial"], case["bcs"], b)
        LC.compare_defined(lab, w, case["labs"][i], case["defined"][i])


def test_oracle_c1_matches_reference_loops(oracle_lib):
    c = c1_small()
    h = c["h"]
    lap = oracle_lib.laplacian_f64(c["comp"], c["nb"], c["n"], {}, (1 / (h * h),) * 3)
    grad = oracle_lib.gradient_f64(c["comp"], c["nb"], c["n"], {}, (1 / h,) * 3)
    assert np.array_equal(lap, c["lap"])
    assert np.array_equal(grad, c["grad"])


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build absent")
def test_oracle_vs_reference_randomised(oracle_lib):
    O = oracle_lib
    rng = np.random.default_rng(7)
    for trial in range(120):
        dt = [np.float64, np.float32, np.int32][trial % 3]
        nb = rng.integers(1, 4, size=3)
        n = rng.integers(2, 7, size=3)
        lo = [int(rng.integers(0, n[d] + 1)) for d in range(3)]
        hi = [int(rng.integers(0, n[d] + 1)) for d in range(3)]
        tens = bool(rng.integers(0, 2))
        nblocks = int(np.prod(nb))
        stride = O.block_stride(n, dt)
        if dt == np.int32:
            comp = rng.integers(-1000, 1000, size=nblocks * stride).astype(dt)
        else:
            comp = (rng.standard_normal(nblocks * stride) * 100).astype(dt)
        bcl = {b: [(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 4)),
                    float(rng.integers(-3, 4))) for _ in range(int(rng.integers(0, 5)))]
               for b in range(nblocks)}
        for block in range(nblocks):
            a, wa = O.lab_fill(comp, nb, n, lo, hi, tens, bcl, block)
            r, wr = O.lab_fill(comp, nb, n, lo, hi, tens, bcl, block, use_ref=True)
            # a symmetry sign of 0 makes the reference define a cell from an
            # undefined one; the oracle calls it undefined
            assert np.all(wa <= wr)
            assert np.array_equal(a[wa], r[wa])


# ---- the reference's unit-test assertions on oracle labs -------------------

def _iota(n, dtype):
    import oracle as O
    a = np.zeros(O.block_stride(n, dtype), dtype=dtype)
    a[: int(np.prod(n))] = np.arange(int(np.prod(n)), dtype=dtype)
    return a


@pytest.mark.parametrize("tens", [False, True])
def test_fieldlab_ghosts(oracle_lib, tens):
    """FieldLabTest.cpp:16-100, DIM 3, Cell."""
    n = (16, 16, 16)
    comp = _iota(n, np.int32)
    lab, w = oracle_lib.lab_fill(comp, (1, 1, 1), n, (2, 2, 2), (2, 2, 2), tens, {}, 0)
    LC.check_fieldlab_ghosts(LC.Lab(lab, n, (2,) * 3, (2,) * 3), comp[: 16 ** 3], tens)


@pytest.mark.parametrize("tens", [False, True])
def test_bc_dirichlet(oracle_lib, tens):
    n = (16,) * 3
    comp = _iota(n, np.int32)
    D = oracle_lib.BC_DIRICHLET
    if not tens:
        bcs = [(0, 0, D, 10), (0, 1, D, 11), (1, 0, D, 12), (1, 1, D, 13), (2, 0, D, 14), (2, 1, D, 15)]
        lab, _ = oracle_lib.lab_fill(comp, (1,) * 3, n, (3,) * 3, (3,) * 3, False, {0: bcs}, 0)
        L = LC.Lab(lab, n, (3,) * 3, (3,) * 3)
        for d, (v0, v1) in enumerate([(10, 11), (12, 13), (14, 15)]):
            LC.check_dirichlet(L, d, v0, v1, False)
    else:
        for d, (v0, v1) in enumerate([(101, 102), (103, 104), (105, 106)]):
            lab, _ = oracle_lib.lab_fill(comp, (1,) * 3, n, (3,) * 3, (3,) * 3, True,
                                         {0: [(d, 0, D, v0), (d, 1, D, v1)]}, 0)
            LC.check_dirichlet(LC.Lab(lab, n, (3,) * 3, (3,) * 3), d, v0, v1, True)


@pytest.mark.parametrize("tens", [False, True])
def test_bc_absorbing(oracle_lib, tens):
    n = (16,) * 3
    comp = _iota(n, np.int32)
    A = oracle_lib.BC_ABSORBING
    for d in range(3):
        lab, _ = oracle_lib.lab_fill(comp, (1,) * 3, n, (3,) * 3, (3,) * 3, tens,
                                     {0: [(d, 0, A, 0), (d, 1, A, 0)]}, 0)
        LC.check_absorbing(LC.Lab(lab, n, (3,) * 3, (3,) * 3), d, tens)


@pytest.mark.parametrize("tens", [False, True])
def test_bc_symmetry(oracle_lib, tens):
    n = (16,) * 3
    comp = _iota(n, np.int32)
    S = oracle_lib.BC_SYMMETRY
    for d in range(3):
        s0, s1 = (1, -1) if not tens else (1, 1)
        lab, _ = oracle_lib.lab_fill(comp, (1,) * 3, n, (3,) * 3, (3,) * 3, tens,
                                     {0: [(d, 0, S, s0), (d, 1, S, s1)]}, 0)
        LC.check_symmetry(LC.Lab(lab, n, (3,) * 3, (3,) * 3), d, s0, s1, tens)


def test_bc_no_stencil_width(oracle_lib):
    """BC/CommonTest.cpp:20-62: a (0,1) stencil leaves the lab untouched."""
    n = (4,) * 3
    comp = _iota(n, np.float64)
    for kind, v in ((oracle_lib.BC_ABSORBING, 0), (oracle_lib.BC_DIRICHLET, 1.0),
                    (oracle_lib.BC_SYMMETRY, 1)):
        lab, w = oracle_lib.lab_fill(comp, (1,) * 3, n, (0,) * 3, (0,) * 3, False, {0: [(0, 0, kind, v)]}, 0)
        assert np.array_equal(lab.ravel(), comp[:64])


def test_cartesian_exact_function(oracle_lib):
    """Grid/CartesianTest.cpp:200-318: multi-block periodic grid, tensorial
    (-2,3), ghosts equal the exact periodic function within 8 eps."""
    import oracle as O
    nb, n = (3, 2, 4), (8, 8, 8)
    h = [1.0 / (nb[i] * n[i]) for i in range(3)]
    stride = O.block_stride(n, np.float64)
    comp = np.zeros(int(np.prod(nb)) * stride)

    def f(x):
        return np.sin(2 * np.pi * x[0]) * np.cos(2 * np.pi * x[1]) * np.sin(2 * np.pi * x[2])

    for b in range(int(np.prod(nb))):
        bi = (b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1]))
        z, y, x = np.meshgrid(*[(np.arange(n[d]) + n[d] * bi[d] + 0.5) * h[d] for d in (2, 1, 0)],
                              indexing="ij")
        comp[b * stride: b * stride + 512] = f((x, y, z)).ravel()
    eps = np.finfo(np.float64).eps
    for b in (0, 5, int(np.prod(nb)) - 1):
        bi = (b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1]))
        lab, _ = oracle_lib.lab_fill(comp, nb, n, (2,) * 3, (2,) * 3, True, {}, b)
        LC.check_exact_function(LC.Lab(lab, n, (2,) * 3, (2,) * 3), bi, h, f, 8 * eps)


def _euler_host_state(nb, n, seed=3):
    import oracle as O
    stride = O.block_stride(n, np.float64)
    nbk = int(np.prod(nb))
    rng = np.random.default_rng(seed)
    U = np.zeros((5, nbk * stride))
    rho = 1.0 + 0.3 * rng.random(nbk * stride)
    vel = (rng.random((3, nbk * stride)) * 2 - 1) * 0.1
    U[0] = rho
    U[1:4] = rho * vel
    U[4] = 2.5 + 0.5 * rho * (vel ** 2).sum(0)
    return U


def _c2_bclists(nb):
    ff = (1.0, 0.0, 0.0, 0.0, 2.5)
    out = []
    for c in range(5):
        d = {}
        for b in range(int(np.prod(nb))):
            bi = (b % nb[0], (b // nb[0]) % nb[1], b // (nb[0] * nb[1]))
            lst = []
            if bi[1] == 0: lst.append((1, 0, 2, 0.0))
            if bi[1] == nb[1] - 1: lst.append((1, 1, 2, 0.0))
            if bi[2] == 0: lst.append((2, 0, 1, ff[c]))
            if bi[2] == nb[2] - 1: lst.append((2, 1, 1, ff[c]))
            if lst: d[b] = lst
        out.append(d)
    return out


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build absent")
@pytest.mark.parametrize("stage", [0, 1, 2, 3])
def test_euler_oracle_lab_matches_reference_fieldlab(oracle_lib, stage):
    """The Euler oracle on its restated lab equals the same math on labs
    loaded by the reference's own FieldLab + BCs (mixed C2-style BCs)."""
    nb, n = (2, 3, 2), (8, 8, 8)
    U = _euler_host_state(nb, n)
    Un = _euler_host_state(nb, n, seed=4)
    bcl = _c2_bclists(nb)
    h = (1 / 16, 1 / 24, 1 / 16)
    want = oracle_lib.euler_stage(U, Un if stage > 1 else None, nb, n, bcl, stage, 1e-3, 1.4, h)
    _, got = oracle_lib.ref_euler_stage(U, Un if stage > 1 else None, nb, n, bcl, stage, 1e-3, 1.4, h)
    assert np.array_equal(got, want)


def test_euler_oracle_constant_state_is_steady(oracle_lib):
    nb, n = (2, 2, 2), (8, 8, 8)
    import oracle as O
    stride = O.block_stride(n, np.float64)
    U = np.zeros((5, 8 * stride))
    U[0], U[4] = 1.0, 2.5
    out = oracle_lib.euler_stage(U, None, nb, n, _c2_bclists(nb), 0, 0.0, 1.4, (1 / 16,) * 3)
    assert not out.any()


def _to_global(a, nb, n, dtype, oracle_lib):
    s = oracle_lib.block_stride(n, dtype)
    cells = int(np.prod(n))
    v = a.reshape(-1, s)[:, :cells].reshape(nb[2], nb[1], nb[0], n[2], n[1], n[0])
    return v.transpose(0, 3, 1, 4, 2, 5).reshape(nb[2] * n[2], nb[1] * n[1], nb[0] * n[0])


def test_mg_oracle_solve_satisfies_the_discrete_equation(oracle_lib):
    """The oracle's multigrid solve reaches 1e-8 and its answer satisfies an
    independent numpy statement of div(k grad p) = f (harmonic face means,
    periodic) to that tolerance."""
    nb, n = (2, 2, 2), (8, 8, 8)
    G = nb[0] * n[0]
    rng = np.random.default_rng(3)
    s = oracle_lib.block_stride(n, np.float32)
    N = int(np.prod(nb)) * s
    kg = np.exp(0.3 * rng.standard_normal((G, G, G)))
    for ax in range(3):
        kg = (np.roll(kg, 1, ax) + kg + np.roll(kg, -1, ax)) / 3.0
    fg = rng.standard_normal((G, G, G))
    fg -= fg.mean()

    def to_blocks(g):
        v = g.reshape(nb[2], n[2], nb[1], n[1], nb[0], n[0]).transpose(0, 2, 4, 1, 3, 5).reshape(-1, int(np.prod(n)))
        out = np.zeros((v.shape[0], s), dtype=np.float32)
        out[:, :v.shape[1]] = v
        return out.reshape(N)
    k, f = to_blocks(kg), to_blocks(fg)
    h = 1.0 / G
    p64, cycles, rel = oracle_lib.mg_solve(k, f, nb, n, h, rtol=1e-8, max_cycles=40)
    assert rel <= 1e-8 and cycles < 40
    p = _to_global(p64, nb, n, np.float64, oracle_lib)
    k32 = _to_global(k, nb, n, np.float32, oracle_lib).astype(np.float64)
    f32 = _to_global(f, nb, n, np.float32, oracle_lib).astype(np.float64)
    Lp = np.zeros_like(p)
    for ax in range(3):
        kp, km = np.roll(k32, -1, ax), np.roll(k32, 1, ax)
        hp, hm = 2 * k32 * kp / (k32 + kp), 2 * km * k32 / (km + k32)
        Lp += hp * (np.roll(p, -1, ax) - p) - hm * (p - np.roll(p, 1, ax))
    Lp /= h * h
    assert np.linalg.norm(f32 - Lp) <= 2e-8 * np.linalg.norm(f32)


ENTITY_N = {1: lambda c: [v + 1 for v in c], 2: lambda c: [c[0] + 1, c[1], c[2]],
            3: lambda c: [c[0], c[1] + 1, c[2]], 4: lambda c: [c[0], c[1], c[2] + 1]}


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build absent")
@pytest.mark.parametrize("entity", [1, 2, 3, 4], ids=["node", "face_x", "face_y", "face_z"])
def test_oracle_vs_reference_node_face(oracle_lib, entity):
    """Node grids and the three face fields of a FaceContainer grid
    (Grid::Cartesian<T, Mesh, EntityType::Node|Face>, where only the last
    block along a grown dimension holds cells + 1 entities): the C oracle
    against the reference's FieldLab on those fields, with randomised
    geometries, stencils and BC vectors."""
    O = oracle_lib
    rng = np.random.default_rng(100 + entity)
    for trial in range(40):
        nb = rng.integers(1, 4, size=3)
        cells = [int(v) for v in rng.integers(2, 6, size=3)]
        n = ENTITY_N[entity](cells)
        lo = [int(rng.integers(0, cells[d] + 1)) for d in range(3)]
        hi = [int(rng.integers(0, cells[d] + 1)) for d in range(3)]
        tens = bool(rng.integers(0, 2))
        nblocks = int(np.prod(nb))
        stride = O.entity_stride(cells, entity, np.float64)
        comp = rng.standard_normal(nblocks * stride) * 100
        bcl = {b: [(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 4)),
                    float(rng.integers(-3, 4))) for _ in range(int(rng.integers(0, 5)))]
               for b in range(nblocks)}
        for block in range(nblocks):
            a, wa = O.lab_fill(comp, nb, n, lo, hi, tens, bcl, block, stride=stride, entity=entity)
            r, wr = O.lab_fill(comp, nb, n, lo, hi, tens, bcl, block, use_ref=True, stride=stride, entity=entity)
            assert np.all(wa <= wr)
            assert np.array_equal(a[wa], r[wa])


@pytest.mark.parametrize("entity", [1, 2], ids=["node", "face_x"])
@pytest.mark.parametrize("tens", [False, True])
def test_node_face_periodic_identities(oracle_lib, entity, tens):
    """FieldLabTest.cpp:56-100 for Node and Face fields (there in 2-D): one
    periodic block, stencil (-2, 3); ghosts equal the values one extent away."""
    O = oracle_lib
    cells = [16, 16, 16]
    n = ENTITY_N[entity](cells)
    stride = O.entity_stride(cells, entity, np.float64)
    comp = np.zeros(stride)
    comp[: int(np.prod(n))] = np.arange(int(np.prod(n)), dtype=np.float64)
    lab, w = O.lab_fill(comp, (1, 1, 1), n, (2, 2, 2), (2, 2, 2), tens, {}, 0, stride=stride, entity=entity)
    f = comp[: int(np.prod(n))].reshape(n[2], n[1], n[0])
    L = LC.Lab(lab, n, (2, 2, 2), (2, 2, 2))
    W = LC.Lab(w, n, (2, 2, 2), (2, 2, 2))
    for z in range(-2, n[2] + 2):
        for y in range(-2, n[1] + 2):
            for x in range(-2, n[0] + 2):
                if not W[(x, y, z)]:
                    continue
                assert L[(x, y, z)] == f[z % n[2], y % n[1], x % n[0]]
