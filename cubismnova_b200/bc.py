"""Boundary conditions (include/Cubism/BC): descriptors pushed into a block
field's BC vector.  The device applies them inside every lab load exactly as
``FieldLab::loadData`` does (Block/FieldLab.h:206-223)."""
from __future__ import annotations

from dataclasses import dataclass

BASE, DIRICHLET, ABSORBING, SYMMETRY = 0, 1, 2, 3


@dataclass(frozen=True)
class BoundaryInfo:
    """BC::BoundaryInfo (BC/Base.h:21-28)."""
    dir: int
    side: int
    is_periodic: bool


class Base:
    """BC::Base (BC/Base.h:39-79): periodic no-op."""
    kind = BASE

    def __init__(self, dir: int, side: int):
        if dir not in (0, 1, 2) or side not in (0, 1):
            raise ValueError("BC: dir must be 0..2 and side 0 or 1")
        self._info = BoundaryInfo(int(dir), int(side), self.kind == BASE)

    def getBoundaryInfo(self) -> BoundaryInfo:
        return self._info

    def name(self) -> str:
        return "Base"

    @property
    def value(self) -> float:
        return 0.0


class Dirichlet(Base):
    """BC::Dirichlet (BC/Dirichlet.h:38-113): ghosts := value."""
    kind = DIRICHLET

    def __init__(self, dir: int, side: int, value: float):
        super().__init__(dir, side)
        self._v = value

    def name(self):
        return "Dirichlet"

    def getValue(self):
        return self._v

    @property
    def value(self):
        return float(self._v)


class Absorbing(Base):
    """BC::Absorbing (BC/Absorbing.h:35-104): zeroth-order extrapolation."""
    kind = ABSORBING

    def name(self):
        return "Zeroth-Order Absorbing"


class Symmetry(Base):
    """BC::Symmetry (BC/Symmetry.h:43-114): ghost := sign * mirrored inner cell."""
    kind = SYMMETRY

    def __init__(self, dir: int, side: int, sign: float = 1):
        super().__init__(dir, side)
        self._s = sign

    def name(self):
        return "Symmetry"

    @property
    def value(self):
        return float(self._s)
