"""Compressible Navier-Stokes RHS (reference: equations/compressible_navier_stokes.py).

`get_rhs_fn(replicas, cfg, physics_models)` returns
`rhs(replica_id, conservative, helper_vars) -> dict`, the same contract as
compressible_navier_stokes.py:46-270: the conservative dict is copied, its
halos filled from `cfg.bc`, and the time derivative of every conserved
variable is returned (valid on interior cells; halo cells are zero). The
whole chain of steps 1-9 (compressible_navier_stokes.py:99-267) runs as one
fused CUDA stage kernel per call (swirlc_b200/csrc/swc_stage.cuh).
"""

import enum
from typing import Dict

import numpy as np
import torch

from swirlc_b200 import engine
from swirlc_b200.boundary import bc_types
from swirlc_b200.common import types
from swirlc_b200.common import utils

_CELL_FACE_BC = bc_types.BoundaryDictionaryType.CELL_FACES.value


class InterpolationSchemes(enum.Enum):
  """compressible_navier_stokes.py:39-43."""
  WENO_3 = 'WENO_3'
  WENO_5 = 'WENO_5'
  MUSCL = 'MUSCL'


class _SolverCache:
  """Solvers keyed by field shape, dtype and device for one cfg."""

  def __init__(self, replicas, cfg, physics_models, interp_override=None):
    self.replicas = replicas
    self.cfg = cfg
    self.pm = physics_models
    self.interp_override = interp_override
    self._cache = {}

  def get(self, replica_id, fields) -> engine.Solver:
    f = fields[0]
    key = (tuple(f.shape), f.dtype, f.device, int(replica_id))
    s = self._cache.get(key)
    if s is None:
      s = engine.Solver(self.cfg, self.pm, f.shape, f.dtype, f.device,
                        replica_id=int(replica_id), replicas=self.replicas,
                        interp_override=self.interp_override)
      self._cache[key] = s
    return s


def _check_cfg(cfg):
  engine.interp_code(cfg)
  engine.riemann_code(cfg)
  if cfg.include_diffusion and _CELL_FACE_BC in cfg.bc:
    raise NotImplementedError(
        'Face boundary conditions are not supported with diffusion enabled at'
        ' this time.')


def _ordered_fields(conservative, cfg=None) -> list:
  """Fields in the solver's order: rho, rho_u, rho_v, rho_w, rho_e, then the
  transported scalars in the order of cfg.conservative_variable_names."""
  missing = [n for n in types.BASE_CONSERVATIVE if n not in conservative]
  if missing:
    raise ValueError(f'Missing conservative variables {missing}.')
  extra = [n for n in conservative if n not in types.BASE_CONSERVATIVE]
  if cfg is not None and extra:
    order = [n for n in cfg.conservative_variable_names if n in extra]
    if set(order) != set(extra):
      raise ValueError(
          f'Transported scalars {extra} are not all in the configuration '
          f'({cfg.conservative_variable_names}).')
    extra = order
  out = []
  for n in list(types.BASE_CONSERVATIVE) + extra:
    t = utils.as_tensor3d(conservative[n])
    if not t.is_cuda:
      raise ValueError(f'Field {n} must be a CUDA tensor.')
    out.append(t.contiguous())
  return out


def helper_states(helper_vars):
  """The hydrostatic reference states when both are given (the reference
  uses them only then, compressible_navier_stokes.py:309)."""
  if helper_vars and 'p_ref' in helper_vars and 'rho_ref' in helper_vars:
    return {'p_ref': utils.as_tensor3d(helper_vars['p_ref']).contiguous(),
            'rho_ref': utils.as_tensor3d(helper_vars['rho_ref']).contiguous()}
  return None


def get_rhs_fn(replicas: np.ndarray, cfg, physics_models):
  """compressible_navier_stokes.py:46-270."""
  _check_cfg(cfg)
  cache = _SolverCache(replicas, cfg, physics_models,
                       getattr(cfg, '_interp_override', None))

  def rhs(replica_id, conservative: Dict, helper_vars: Dict) -> Dict:
    fields = _ordered_fields(conservative, cfg)
    solver = cache.get(replica_id, fields)
    out = solver.rhs(fields, helper_states(helper_vars))
    res = dict(zip(solver.names, out))
    return {k: utils.like_input(res[k], conservative[k]) for k in conservative}

  rhs._swc_cache = cache  # lets rk3/rk2 run the fused in-place stages
  return rhs


def _compute_physical_flux_1d(conservative: Dict, primitive: Dict,
                              helper_var: Dict, dim: str,
                              conservative_var_name: str):
  """compressible_navier_stokes.py:338-427: the physical convective flux.

  Mass flux rho*u_dim; momentum aligned with `dim`: rho*u_dim*u_dim + p (p_dyn
  when the helper variable is present); energy: rho*u_dim*(e + p/rho) with the
  full p; other conserved variables: rho*u_dim*phi. This is the flux the
  fused stage and the pointwise Riemann kernel compute on the device; the
  function is the reference's `flux_fn` argument of hll/hllc_convective_flux
  and evaluates with torch operations on whatever tensors it is given.
  """
  p_updated = helper_var.get('p_dyn', primitive[types.P]) if helper_var \
      else primitive[types.P]
  var = types.conservative_to_primitive_name(conservative_var_name)
  aligned_vel = types.VELOCITY[types.DIMS.index(dim)]
  aligned_mom = types.primitive_to_conservative_name(aligned_vel)
  m = conservative[aligned_mom]
  if var == aligned_vel:
    return m * primitive[aligned_vel] + p_updated
  if var == types.E:
    return m * (primitive[types.E] + primitive[types.P] / primitive[types.RHO])
  if var == types.RHO:
    return m
  return m * primitive[var]


def _intercell_diffusive_flux(primitive: Dict, cfg, physics_models) -> Dict:
  """compressible_navier_stokes.py:618-707: the diffusive flux across every
  face i-1/2 of every conserved variable: 0 for rho and transported
  scalars, -tau_{i,dim} for rho_u_i, q_dim - u_f . tau_{.,dim} for rho_e;
  computed by the fused stage's viscous face routine (swc_viscous_terms)."""
  from swirlc_b200 import _native as nat
  from swirlc_b200.numerics import _pointwise
  tm = physics_models.transport_model
  out = _pointwise.viscous_terms(nat.SWC_VISC_FLUX, primitive, cfg,
                                 nu=tm.nu, pr=tm.pr)
  names = list(getattr(cfg, 'conservative_variable_names',
                       types.BASE_CONSERVATIVE))
  ref = primitive[types.RHO]
  base = dict(zip(types.BASE_CONSERVATIVE, range(5)))
  res = {}
  for d, dim in enumerate(types.DIMS):
    res[dim] = {}
    for name in names:
      if name in base:
        res[dim][name] = utils.like_input(out[d * 5 + base[name]], ref)
      else:
        res[dim][name] = utils.like_input(torch.zeros_like(out[d * 5]), ref)
  return res
