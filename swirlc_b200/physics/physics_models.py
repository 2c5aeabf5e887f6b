"""Physics model container (reference: physics/physics_models.py:27-143).

Selects the thermodynamics, transport and source models exactly as the
reference and raises the same errors for unknown names. The model objects
carry configuration only; their arithmetic runs inside the CUDA kernels.
"""

import enum

from swirlc_b200.common import types
from swirlc_b200.physics.additional_models import gravity
from swirlc_b200.physics.thermodynamics import generic
from swirlc_b200.physics.transport import simple


class ThermodynamicsModels(enum.Enum):
  GENERIC = 'generic'


class TransportModels(enum.Enum):
  SIMPLE = 'simple'


class SourceTermModels(enum.Enum):
  GRAVITY = 'gravity'


class PhysicsModels:
  """physics_models.py:42-143."""

  def __init__(self, cfg):
    if cfg.thermodynamics_model == ThermodynamicsModels.GENERIC.value:
      self.thermodynamics_model = generic.ThermodynamicsGeneric()
    else:
      raise NotImplementedError(
          'Unsupported thermodynamics model:'
          f' "{cfg.thermodynamics_model}". Supported models are: '
          + str([m.value for m in ThermodynamicsModels]))
    if cfg.transport_model == TransportModels.SIMPLE.value:
      self.transport_model = simple.TransportSimple(cfg)
    else:
      raise NotImplementedError(
          'Unsupported transport model:'
          f' "{cfg.transport_model}". Supported models are: '
          + str([m.value for m in TransportModels]))
    self.source_functions = []
    if cfg.source_functions:
      for name in cfg.source_functions:
        if name == SourceTermModels.GRAVITY.value:
          self.source_functions.append(gravity.Gravity(cfg))
        else:
          raise NotImplementedError(
              f'Unsupported source term model: "{name}".'
              ' Supported models are: '
              + str([m.value for m in SourceTermModels]))

  def gravity_mask(self) -> int:
    """Bit d set when rho_u_d receives the gravity source (gravity.py:51-62)."""
    mask = 0
    for model in self.source_functions:
      for name in model.mask():
        mask |= 1 << types.MOMENTUM.index(name)
    return mask
