"""Numerical flux selection (reference: riemann_solver.py:24-62)."""

import enum

from swirlc_b200.numerics.riemann_solver import hll
from swirlc_b200.numerics.riemann_solver import hllc


class NumericFluxScheme(enum.Enum):
  HLL = 'HLL'
  HLLC = 'HLLC'


def select_numeric_flux_fn(cfg):
  """riemann_solver.py:30-62."""
  if cfg.numeric_flux_scheme == NumericFluxScheme.HLL.value:
    return hll.hll_convective_flux
  if cfg.numeric_flux_scheme == NumericFluxScheme.HLLC.value:
    return hllc.hllc_convective_flux
  raise ValueError(
      f'"{cfg.numeric_flux_scheme}" is not implemented as a'
      ' "numeric_flux_scheme". Valid options are: '
      + str([s.value for s in NumericFluxScheme]))
