"""Diffusive terms (reference: physics/diffusion.py).

shear_stress and single_component_heat_flux run the viscous face routine of
the fused stage kernel as a unit-level CUDA kernel (swc_viscous_terms), so
they return exactly the stress and heat flux the stage applies. Face index i
holds face i-1/2; faces whose stencil leaves the array hold 0.
"""

from typing import Dict, List

from swirlc_b200 import _native as nat
from swirlc_b200.common import types
from swirlc_b200.common import utils
from swirlc_b200.numerics import _pointwise


def shear_stress(states: Dict, states_fx: Dict, states_fy: Dict,
                 states_fz: Dict, cfg, physics_models) -> List[List]:
  """diffusion.py:33-67: tau_ij = 2 rho_j nu S_ij on the j faces, with the
  face densities rho_j of states_fx/fy/fz and nu of the transport model."""
  nu = physics_models.transport_model.nu
  out = _pointwise.viscous_terms(
      nat.SWC_VISC_STRESS, states, cfg,
      rho_face=[states_fx[types.RHO], states_fy[types.RHO],
                states_fz[types.RHO]], nu=nu, pr=1.0)
  ref = states[types.U]
  return [[utils.like_input(out[i * 3 + j], ref) for j in range(3)]
          for i in range(3)]


def single_component_heat_flux(primitive: Dict, cfg,
                               physics_models) -> Dict[str, object]:
  """diffusion.py:76-109: -kappa_f dT/dx_j on the j faces, T = p/(rho R),
  kappa = cp nu rho / pr linearly interpolated to the face."""
  tm = physics_models.transport_model
  out = _pointwise.viscous_terms(nat.SWC_VISC_HEAT, primitive, cfg,
                                 nu=tm.nu, pr=tm.pr)
  ref = primitive[types.RHO]
  return {d: utils.like_input(out[i], ref) for i, d in enumerate(types.DIMS)}
