"""hydro3d_b200 -- B200-native pressure-Poisson multigrid for Hydro3D's projection step.

The product is the C-ABI library libh3dmg.so (include/h3d_mg.h) built from
hydro3d_b200/csrc for sm_100a; this package is its host-side mirror.
"""
from ._lib import H3DError, lib  # noqa: F401
from .mg import MultigridSolver, halo_table, host_field, interior, with_ghost  # noqa: F401
from . import topology  # noqa: F401

__all__ = ["MultigridSolver", "H3DError", "halo_table", "host_field", "interior", "with_ghost", "topology", "lib"]
