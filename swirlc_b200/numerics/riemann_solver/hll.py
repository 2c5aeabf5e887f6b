"""HLL numerical flux (reference: numerics/riemann_solver/hll.py).

hll_convective_flux evaluates hll.py:107-170 with the physical flux of
compressible_navier_stokes.py:338-427 in one pointwise CUDA kernel
(swc_riemann_flux). `flux_fn` is accepted for signature compatibility; the
physical flux is the reference's own (_compute_physical_flux_1d).
"""

from swirlc_b200 import _native as nat
from swirlc_b200.numerics import _pointwise


def hll_convective_flux(replica_id, replicas, conservative_neg,
                        conservative_pos, primitive_neg, primitive_pos,
                        helper_var_neg, helper_var_pos, flux_fn, dim, cfg,
                        physics_models):
  """hll.py:36-175."""
  del flux_fn, physics_models
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
