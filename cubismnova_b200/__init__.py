"""cubismnova_b200 -- B200-native CubismNova lab fill + stencil hot path.

Host-side mirror of the reference API for this path (namespaces ``Core``,
``Grid``, ``Block``, ``BC``, ``IO`` and the stencil operators in ``ops``) over the C
ABI of ``libcubismnova_b200.so``.  Names, argument meaning and error messages
follow CubismNova (``include/Cubism/...``); all data lives on the GPU.
"""
from . import _lib
from ._lib import CnError, build
from . import core as Core
from . import bc as BC
from . import grid as Grid
from . import block as Block
from . import ops
from . import euler
from . import workloads
from . import mg
from . import learned
from . import amr
from . import io as IO
from . import partition

__all__ = ["Core", "BC", "Grid", "Block", "ops", "euler", "workloads", "mg", "learned", "amr", "IO", "partition", "CnError", "build"]
