"""Time integration dispatcher (reference: time_integration.py:27-90)."""

import enum

from swirlc_b200.numerics.time_integration import rk2
from swirlc_b200.numerics.time_integration import rk3


class TimeIntegrationScheme(enum.Enum):
  RK2 = 'rk2'
  RK3 = 'rk3'


def time_integration(replica_id, replicas, state_0, helper_vars, cfg,
                     physics_models, rhs_fn):
  """time_integration.py:35-90."""
  if cfg.time_integration_scheme == TimeIntegrationScheme.RK3.value:
    return rk3.integrate(replica_id, replicas, state_0, helper_vars, cfg,
                         physics_models, rhs_fn)
  if cfg.time_integration_scheme == TimeIntegrationScheme.RK2.value:
    return rk2.integrate(replica_id, replicas, state_0, helper_vars, cfg,
                         physics_models, rhs_fn)
  raise NotImplementedError(
      f'"{cfg.time_integration_scheme}" is not implemented as an'
      ' "time_integration_scheme". Valid options are: '
      + str([s.value for s in TimeIntegrationScheme]))
