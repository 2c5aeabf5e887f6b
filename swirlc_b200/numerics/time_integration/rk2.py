"""Second-order Runge-Kutta (reference: numerics/time_integration/rk2.py).

u1 = u0 + dt L(u0); u2 = u1 + dt L(u1); u_n = 0.5 (u0 + u2) (rk2.py:63-86).
"""

from swirlc_b200 import _native as nat
from swirlc_b200.numerics.time_integration import _stages


def integrate(replica_id, replicas, state_0, helper_vars, cfg, physics_models,
              rhs_fn):
  """rk2.py:30-86."""
  del replicas, physics_models
  cache = getattr(rhs_fn, '_swc_cache', None)
  if cache is not None:
    from swirlc_b200.equations import compressible_navier_stokes as cns
    from swirlc_b200.common import utils
    fields = cns._ordered_fields(state_0, cfg)
    solver = cache.get(replica_id, fields)
    out = solver.rk2(fields, cfg.dt, cns.helper_states(helper_vars))
    res = dict(zip(solver.names, out))
    return {k: utils.like_input(res[k], state_0[k]) for k in state_0}
  dt_t = _stages.dt_tensor(cfg.dt, _stages.first_device(state_0))
  df = rhs_fn(replica_id, state_0, helper_vars)
  s1 = {k: _stages.combine(nat.SWC_OUT_EULER, 0, 0, dt_t, None, v, df[k])
        for k, v in state_0.items()}
  df = rhs_fn(replica_id, s1, helper_vars)
  return {k: _stages.combine(nat.SWC_OUT_AVERAGE, 0.5, 0.0, dt_t, v, s1[k],
                             df[k])
          for k, v in state_0.items()}
