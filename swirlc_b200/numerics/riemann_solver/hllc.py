"""HLLC numerical flux (reference: numerics/riemann_solver/hllc.py)."""

from swirlc_b200 import _native as nat
from swirlc_b200.common import types
from swirlc_b200.numerics import _pointwise


def hllc_convective_flux(replica_id, replicas, conservative_neg,
                         conservative_pos, primitive_neg, primitive_pos,
                         helper_var_neg, helper_var_pos, flux_fn, dim, cfg,
                         physics_models):
  """hllc.py:33-257 (pointwise CUDA kernel swc_riemann_flux)."""
  del physics_models
  _pointwise.check_flux_fn(flux_fn, list(getattr(
      cfg, 'conservative_variable_names', types.BASE_CONSERVATIVE)))
  return _pointwise.riemann_flux(nat.SWC_HLLC, conservative_neg,
                                 conservative_pos, primitive_neg,
                                 primitive_pos, helper_var_neg, helper_var_pos,
                                 dim, cfg, replica_id, replicas)


def _compute_wave_speeds(replica_id, replicas, primitive_neg, primitive_pos,
                         dim, cfg, physics_models):
  """hllc.py:260-347: (s_l, s_m, s_r)."""
  del physics_models
  return _pointwise.wave_speeds(primitive_neg, primitive_pos, dim, cfg, True,
                                replica_id, replicas)
