"""Core::Stencil and a minimal Core::IndexRange (include/Cubism/Core)."""
from __future__ import annotations

from . import _lib


def _vec3(v):
    if isinstance(v, (int,)):
        return (int(v),) * 3
    t = tuple(int(x) for x in v)
    if len(t) != 3:
        raise ValueError("expected 3 components")
    return t


class IndexRange:
    """Core::IndexRange<3> subset (Core/Index.h:130-310): [begin, end), x fastest."""

    def __init__(self, begin_or_extent, end=None):
        if end is None:
            self._b, self._e = (0, 0, 0), _vec3(begin_or_extent)
        else:
            self._b, self._e = _vec3(begin_or_extent), _vec3(end)

    def getBegin(self):
        return self._b

    def getEnd(self):
        return self._e

    def getExtent(self):
        return tuple(e - b for b, e in zip(self._b, self._e))

    def size(self):
        x, y, z = self.getExtent()
        return x * y * z

    def isIndex(self, p):
        return all(b <= v < e for b, v, e in zip(self._b, p, self._e))

    def __iter__(self):
        (b0, b1, b2), (e0, e1, e2) = self._b, self._e
        for z in range(b2, e2):
            for y in range(b1, e1):
                for x in range(b0, e0):
                    yield (x, y, z)

    def __eq__(self, o):
        return isinstance(o, IndexRange) and self._b == o._b and self._e == o._e

    def __repr__(self):
        return f"IndexRange({self._b}, {self._e})"


class Stencil:
    """Core::Stencil (Core/Stencil.h:21-108).

    ``Stencil(-1, 2)`` is the symmetric 3-point stencil; ``end`` is exclusive.
    Raises RuntimeError("Stencil: begin_ must be <= 0") /
    ("Stencil: end_ must be > 0") exactly where the reference throws; in
    addition a single violating component is rejected (the device lab cannot
    represent it).
    """

    def __init__(self, begin=0, end=1, tensorial=False):
        self._b = _vec3(begin)
        self._e = _vec3(end)
        self._t = bool(tensorial)
        s = self.as_struct()
        _lib.check(_lib.lib().cn_stencil_check(s))

    def getBegin(self):
        return self._b

    def getEnd(self):
        return self._e

    def isTensorial(self):
        return self._t

    def as_struct(self):
        return _lib.stencil_struct(self._b, self._e, self._t)

    def __eq__(self, o):
        return isinstance(o, Stencil) and (self._b, self._e, self._t) == (o._b, o._e, o._t)

    def __repr__(self):
        return f"Stencil({self._b}, {self._e}, tensorial={self._t})"
