"""Third-order SSP Runge-Kutta (reference: numerics/time_integration/rk3.py).

u1 = u0 + dt L(u0); u2 = c11 u0 + c12 (u1 + dt L(u1));
u_n = c21 u0 + c22 (u2 + dt L(u2)) with the coefficients of rk3.py:24-31.
When `rhs_fn` comes from `get_rhs_fn`, each stage is one fused CUDA pass
(halo fill + RHS + combination); any other rhs callable is evaluated as
given and combined by the swc_rk_combine kernel.
"""

from swirlc_b200 import _native as nat
from swirlc_b200.numerics.time_integration import _stages

_RK3_COEFFS = {'c11': 0.75, 'c21': 1.0 / 3.0}
_RK3_COEFFS['c12'] = 1.0 - _RK3_COEFFS['c11']
_RK3_COEFFS['c22'] = 1.0 - _RK3_COEFFS['c21']


def integrate(replica_id, replicas, state_0, helper_vars, cfg, physics_models,
              rhs_fn):
  """rk3.py:34-122."""
  del replicas, physics_models
  cache = getattr(rhs_fn, '_swc_cache', None)
  if cache is not None:
    from swirlc_b200.equations import compressible_navier_stokes as cns
    from swirlc_b200.common import utils
    fields = cns._ordered_fields(state_0, cfg)
    solver = cache.get(replica_id, fields)
    out = solver.rk3(fields, cfg.dt, cns.helper_states(helper_vars))
    res = dict(zip(solver.names, out))
    return {k: utils.like_input(res[k], state_0[k]) for k in state_0}
  dt_t = _stages.dt_tensor(cfg.dt, _stages.first_device(state_0))
  df = rhs_fn(replica_id, state_0, helper_vars)
  s1 = {k: _stages.combine(nat.SWC_OUT_EULER, 0, 0, dt_t, None, v, df[k])
        for k, v in state_0.items()}
  df = rhs_fn(replica_id, s1, helper_vars)
  s2 = {k: _stages.combine(nat.SWC_OUT_CONVEX, _RK3_COEFFS['c11'],
                           _RK3_COEFFS['c12'], dt_t, v, s1[k], df[k])
        for k, v in state_0.items()}
  df = rhs_fn(replica_id, s2, helper_vars)
  return {k: _stages.combine(nat.SWC_OUT_CONVEX, _RK3_COEFFS['c21'],
                             _RK3_COEFFS['c22'], dt_t, v, s2[k], df[k])
          for k, v in state_0.items()}
