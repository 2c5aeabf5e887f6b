"""HLL numerical flux (reference: numerics/riemann_solver/hll.py).

hll_convective_flux evaluates hll.py:107-170 with the physical flux of
compressible_navier_stokes.py:338-427 in one pointwise CUDA kernel
(swc_riemann_flux). `flux_fn` must be None or compute that physical flux
(_compute_physical_flux_1d); any other function raises NotImplementedError.
"""

from swirlc_b200 import _native as nat
from swirlc_b200.common import types
from swirlc_b200.numerics import _pointwise


def hll_convective_flux(replica_id, replicas, conservative_neg,
                        conservative_pos, primitive_neg, primitive_pos,
                        helper_var_neg, helper_var_pos, flux_fn, dim, cfg,
                        physics_models):
  """hll.py:36-175."""
  del physics_models
  _pointwise.check_flux_fn(flux_fn, list(getattr(
      cfg, 'conservative_variable_names', types.BASE_CONSERVATIVE)))
  return _pointwise.riemann_flux(nat.SWC_HLL, conservative_neg,
                                 conservative_pos, primitive_neg,
                                 primitive_pos, helper_var_neg, helper_var_pos,
                                 dim, cfg, replica_id, replicas)


def compute_hll_roe_wave_speed_estimates(replica_id, replicas, primitive_neg,
                                         primitive_pos, dim, cfg,
                                         physics_models):
  """hll.py:178-283: (s_l, s_r)."""
  del physics_models
  return _pointwise.wave_speeds(primitive_neg, primitive_pos, dim, cfg, False,
                                replica_id, replicas)
