"""Simulation step (reference: core/simulation.py:27-105)."""

import enum

import numpy as np

from swirlc_b200.equations import compressible_navier_stokes
from swirlc_b200.numerics.time_integration import time_integration
from swirlc_b200.physics import physics_models as physics_models_lib


class Solvers(enum.Enum):
  COMPRESSIBLE_NS = 'compressible_navier_stokes'


class Simulation:
  """simulation.py:32-105."""

  def __init__(self, kernel_op, cfg):
    del kernel_op  # Unused, as in the reference.
    self.cfg = cfg
    self.physics_models = physics_models_lib.PhysicsModels(cfg)
    shape = np.array([cfg.cx, cfg.cy, cfg.cz])
    replicas = np.arange(np.prod(shape), dtype=np.int32).reshape(shape)
    if cfg.solver == Solvers.COMPRESSIBLE_NS.value:
      self.rhs_fn = compressible_navier_stokes.get_rhs_fn(
          replicas, self.cfg, self.physics_models)
    else:
      raise NotImplementedError(
          f'"{cfg.solver}" is not an implemented solver. Valid options are: '
          '"compressible_navier_stokes"')

  def step(self, replica_id, replicas, step_id, states, additional_states):
    """simulation.py:68-105."""
    del step_id
    return time_integration.time_integration(
        replica_id, replicas, states, additional_states, self.cfg,
        self.physics_models, self.rhs_fn)
