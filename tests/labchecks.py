"""Assertions of the reference's unit tests, re-expressed on a dense lab array.

A lab is indexed lab[z+lo2, y+lo1, x+lo0] for lab cell (x, y, z); the helpers
below take lab cell coordinates.  Used by the oracle tests (CPU) and by the
device tests (GPU) alike.
"""
import numpy as np


class Lab:
    def __init__(self, arr, n, lo, hi):
        self.a, self.n, self.lo, self.hi = arr, tuple(n), tuple(lo), tuple(hi)

    def __getitem__(self, p):
        x, y, z = p
        return self.a[z + self.lo[2], y + self.lo[1], x + self.lo[0]]

    def lab_range(self):
        lo, hi, n = self.lo, self.hi, self.n
        for z in range(-lo[2], n[2] + hi[2]):
            for y in range(-lo[1], n[1] + hi[1]):
                for x in range(-lo[0], n[0] + hi[0]):
                    yield (x, y, z)


def unit(i, s=1):
    v = [0, 0, 0]
    v[i] = s
    return v


def check_fieldlab_ghosts(lab: Lab, field, tensorial: bool):
    """test/UnitTests/Block/FieldLabTest.cpp:53-99 (self-periodic field)."""
    n = lab.n
    f = field.reshape(n[2], n[1], n[0])
    for z in range(n[2]):
        for y in range(n[1]):
            for x in range(n[0]):
                assert lab[(x, y, z)] == f[z, y, x]
    if not tensorial:
        for z in range(n[2]):
            for y in range(n[1]):
                for x in range(n[0]):
                    p = (x, y, z)
                    for i in range(3):
                        if p[i] == 0:
                            for si in range(-lab.lo[i], 0):
                                sm = list(p); sm[i] += si
                                sp = list(p); sp[i] += si + n[i]
                                assert lab[sm] == lab[sp]
                        if p[i] == n[i] - 1:
                            for si in range(1, lab.hi[i] + 1):
                                sm = list(p); sm[i] += si - n[i]
                                sp = list(p); sp[i] += si
                                assert lab[sm] == lab[sp]
    else:
        for q in lab.lab_range():
            if all(0 <= q[i] < n[i] for i in range(3)):
                continue
            s = [q[i] + n[i] if q[i] < 0 else (q[i] % n[i] if q[i] >= n[i] else q[i]) for i in range(3)]
            assert lab[q] == lab[s]


def _slab(lab: Lab, d, side, tensorial):
    """Cells of the ghost slab (d, side) as the BC tests iterate them."""
    n, lo, hi = lab.n, lab.lo, lab.hi
    rng = []
    for i in range(3):
        if i == d:
            rng.append(range(-lo[i], 0) if side == 0 else range(n[i], n[i] + hi[i]))
        elif tensorial:
            rng.append(range(-lo[i], n[i] + hi[i]))
        else:
            rng.append(range(0, n[i]))
    for z in rng[2]:
        for y in rng[1]:
            for x in rng[0]:
                yield (x, y, z)


def check_dirichlet(lab: Lab, d, v0, v1, tensorial):
    """test/UnitTests/BC/DirichletTest.cpp:91-110."""
    for q in _slab(lab, d, 0, tensorial):
        assert lab[q] == v0
    for q in _slab(lab, d, 1, tensorial):
        assert lab[q] == v1


def check_absorbing(lab: Lab, d, tensorial):
    """test/UnitTests/BC/AbsorbingTest.cpp: every ghost layer equals the
    adjacent inner layer (zeroth-order extrapolation)."""
    for side in (0, 1):
        for q in _slab(lab, d, side, tensorial):
            src = list(q)
            src[d] = 0 if side == 0 else lab.n[d] - 1
            assert lab[q] == lab[src]


def check_symmetry(lab: Lab, d, s0, s1, tensorial):
    """test/UnitTests/BC/SymmetryTest.cpp:16-45: lab[q] == s * lab[off - q]."""
    for side, s, off in ((0, s0, -1), (1, s1, 2 * lab.n[d] - 1)):
        for q in _slab(lab, d, side, tensorial):
            r = list(q)
            r[d] = off - r[d]
            assert lab[q] == s * lab[r]


def check_exact_function(lab: Lab, block_index, h, fexact, tol):
    """test/UnitTests/Grid/CartesianTest.cpp:245-257: every lab cell (ghosts
    included) equals the periodic exact function within tol."""
    n = lab.n
    for q in lab.lab_range():
        x = [(block_index[i] * n[i] + q[i] + 0.5) * h[i] for i in range(3)]
        assert abs(lab[q] - fexact(x)) <= tol, (q, lab[q], fexact(x))


def compare_defined(got, got_def, want, want_def):
    """Device/oracle lab vs expected: identical on every cell both define, and
    the device defines everything the expectation defines."""
    assert got.shape == want.shape
    both = got_def & want_def
    assert np.array_equal(got_def, want_def), "defined-cell masks differ"
    g, w = got[both], want[both]
    if g.dtype.kind == "f":
        assert np.array_equal(g.view(np.uint8), w.view(np.uint8)), \
            f"{np.sum(g != w)} cells differ (max |diff| {np.max(np.abs(g - w)) if g.size else 0})"
    else:
        assert np.array_equal(g, w), f"{np.sum(g != w)} cells differ"
