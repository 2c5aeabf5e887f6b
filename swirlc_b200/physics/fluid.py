"""Fluid kinematics (reference: physics/fluid.py).

strain_rate runs the viscous face routine of the fused stage kernel as a
unit-level CUDA kernel (swc_viscous_terms). Face index i holds face i-1/2;
faces whose stencil leaves the array hold 0.
"""

from typing import Dict, List

from swirlc_b200 import _native as nat
from swirlc_b200.common import types
from swirlc_b200.common import utils
from swirlc_b200.numerics import _pointwise


def strain_rate(states: Dict, cfg) -> List[List]:
  """fluid.py:31-111: S_ij = (d_j u_i + d_i u_j)/2 - div(u)/3 delta_ij on
  the j faces; the derivative along j is the backward difference, the
  others central differences at the cells linearly interpolated to the
  face."""
  out = _pointwise.viscous_terms(nat.SWC_VISC_STRAIN, states, cfg, nu=0.5,
                                 pr=1.0)
  ref = states[types.U]
  return [[utils.like_input(out[i * 3 + j], ref) for j in range(3)]
          for i in range(3)]
