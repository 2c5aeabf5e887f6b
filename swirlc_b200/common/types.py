"""Names and basic types (reference: common/types.py:14-142).

Variable names, the dimension tuple and the name conversions are the same
strings and rules as the reference, so configs and state dicts written for
the reference work unchanged.
"""

import re
from typing import Dict, List, Sequence, Union

import numpy as np
import torch

# Precision (types.py:24-28). torch replaces tf as the tensor type.
DTYPE = torch.float32
NP_DTYPE = np.float32
SMALL = np.finfo(np.float32).resolution

FlowFieldVar = Union[Sequence[torch.Tensor], torch.Tensor]
MutableFlowFieldVar = List[torch.Tensor]
FlowFieldMap = Dict[str, FlowFieldVar]

DIMS = ('x', 'y', 'z')

RHO = 'rho'
U = 'u'
V = 'v'
W = 'w'
VELOCITY = (U, V, W)
E = 'e'
BASE_PRIMITIVES = (RHO, U, V, W, E)
CONS_VAR_PREFIX = 'rho_'
RHO_U = CONS_VAR_PREFIX + U
RHO_V = CONS_VAR_PREFIX + V
RHO_W = CONS_VAR_PREFIX + W
MOMENTUM = (RHO_U, RHO_V, RHO_W)
RHO_E = CONS_VAR_PREFIX + E
BASE_CONSERVATIVE = (RHO, RHO_U, RHO_V, RHO_W, RHO_E)
P = 'p'
T = 't'
POTENTIAL_T = 'theta'
H = 'h'


def primitive_to_conservative_name(primitive: str) -> str:
  """types.py:82-99."""
  if not primitive:
    raise ValueError('Primitive variable name must not be empty.')
  if primitive == RHO:
    return RHO
  return CONS_VAR_PREFIX + primitive


def conservative_to_primitive_name(conservative: str) -> str:
  """types.py:102-126."""
  if conservative == RHO:
    return RHO
  if is_conservative_name(conservative):
    return conservative[len(CONS_VAR_PREFIX):]
  raise ValueError(
      f'Invalid conserved variable name: {conservative}. Must start with'
      f' "{CONS_VAR_PREFIX}".')


def is_conservative_name(varname: str) -> bool:
  """types.py:129-142."""
  return bool(re.match(f'^({CONS_VAR_PREFIX}).', varname))
