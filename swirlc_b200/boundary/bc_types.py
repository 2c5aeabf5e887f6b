"""Boundary condition types (reference: boundary/bc_types.py:22-47)."""

import enum
from typing import Any, Dict, Tuple


class BoundaryCondition(enum.Enum):
  """Defines the types of the boundary condition."""
  PERIODIC = 0
  DIRICHLET = 1
  NEUMANN = 2
  REFLECTIVE = 3


class BoundaryFluxType(enum.Enum):
  """Defines the different boundary fluxes which can be specified."""
  CONVECTIVE = 'convective'
  DIFFUSIVE = 'diffusive'
  TOTAL = 'total'


class BoundaryDictionaryType(enum.Enum):
  """Defines the location and type of the boundary dictionary."""
  CELL_AVERAGES = 'cell_averages'
  CELL_FACES = 'cell_faces'
  INTERCELL_FLUXES = 'intercell_fluxes'


BCDict = Dict[str, Dict[int, Tuple[BoundaryCondition, Any]]]


def bc_value(bc_type) -> int:
  """Integer value of a BoundaryCondition from this module, the reference's
  identically valued enum, or a plain int."""
  return int(getattr(bc_type, 'value', bc_type))
