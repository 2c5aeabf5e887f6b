"""Gravity source model (reference: physics/additional_models/gravity.py:26-102).

The source d_rho * G * g[dim] is added inside the fused stage kernel to the
momentum components listed by `mask()`.
"""

from swirlc_b200.common import types
from swirlc_b200.common import utils


class Gravity:

  def __init__(self, cfg):
    if utils.gravity_direction(cfg) == -1:
      raise ValueError(
          'Gravity direction must be specified if the gravity source function'
          ' is to be used.')
    self._cfg = cfg

  def mask(self):
    idx = utils.gravity_direction(self._cfg)
    if idx == 3:
      return types.MOMENTUM
    return (types.MOMENTUM[idx],)
