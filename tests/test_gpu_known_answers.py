"""GPU: the CUDA path against more of the reference's own known answers.

The viscous terms run through swc_viscous_terms, which evaluates the fused
stage's own viscous face routine, so these pin the stage's arithmetic:
fluid.strain_rate (fluid_test.py:122-145), diffusion.shear_stress and
single_component_heat_flux (diffusion_test.py:116-201), and
_intercell_diffusive_flux (compressible_navier_stokes_test.py:1979-2102).
The standing Mach-6 shock (:624-775) runs through hll/hllc_convective_flux.
The heat-conduction case also runs through the fused RHS with identity face
values (the reference tests' WENO mock), where the only non-zero time
derivative is -d(q)/dx of rho_e. Tolerances are the reference tests'.
"""

import numpy as np
import pytest
import torch

from oracle import swirlc_oracle as orc
from tests import known_answers as ka

pytestmark = pytest.mark.gpu
DIMS = ('x', 'y', 'z')
NAMES6 = list(orc.BASE_CONSERVATIVE) + ['rho_y']
WIN = (slice(3, -2),) * 3


def _cfg(**kw):
  from swirlc_b200.core import parameter
  return parameter.SwirlCParameters(kw)


def _pm(cfg):
  from swirlc_b200.physics import physics_models
  return physics_models.PhysicsModels(cfg)


def _dev(d, dtype=torch.float64):
  return {k: torch.tensor(np.asarray(v), dtype=dtype, device='cuda')
          for k, v in d.items()}


def _np(t):
  return t.double().cpu().numpy()


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_strain_rate_taylor_green(dtype):
  from swirlc_b200.physics import fluid
  states, expected, delta = ka.strain_rate_case()
  cfg = _cfg(dx=delta['x'], dy=delta['y'], dz=delta['z'])
  s = fluid.strain_rate(_dev(states, dtype), cfg)
  inner = (slice(1, -1),) * 3
  for i in range(3):
    for j in range(3):
      np.testing.assert_allclose(_np(s[i][j])[inner], expected[i][j][inner],
                                 atol=5e-2, rtol=1e-6, err_msg=f'S{i}{j}')


def test_strain_rate_equals_oracle():
  from swirlc_b200.physics import fluid
  states, _, delta = ka.strain_rate_case()
  cfg = _cfg(dx=delta['x'], dy=delta['y'], dz=delta['z'])
  s = fluid.strain_rate(_dev(states), cfg)
  want = orc.strain_rate(states, delta)
  inner = (slice(1, -1),) * 3
  for i in range(3):
    for j in range(3):
      np.testing.assert_allclose(_np(s[i][j])[inner], want[i][j][inner],
                                 rtol=1e-12, atol=1e-12, err_msg=f'S{i}{j}')


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_shear_stress_taylor_green(dtype):
  from swirlc_b200.physics import diffusion
  states, rho_f, expected, delta, nu = ka.shear_stress_case()
  cfg = _cfg(dx=delta['x'], dy=delta['y'], dz=delta['z'],
             transport_parameters={'nu': nu, 'pr': 0.7})
  fx, fy, fz = ({'rho': torch.tensor(rho_f[d], dtype=dtype, device='cuda')}
                for d in DIMS)
  tau = diffusion.shear_stress(_dev(states, dtype), fx, fy, fz, cfg, _pm(cfg))
  inner = (slice(1, -1),) * 3
  for i in range(3):
    for j in range(3):
      np.testing.assert_allclose(_np(tau[i][j])[inner], expected[i][j][inner],
                                 atol=1e-2, rtol=1e-6, err_msg=f'tau{i}{j}')


@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_single_component_heat_flux(dtype):
  from swirlc_b200.physics import diffusion
  prim, expected, delta, nu, pr = ka.heat_flux_case()
  cfg = _cfg(dx=delta['x'], dy=delta['y'], dz=delta['z'],
             transport_parameters={'nu': nu, 'pr': pr})
  q = diffusion.single_component_heat_flux(_dev(prim, dtype), cfg, _pm(cfg))
  # float32: the reference's own test notes large round-off of the
  # T = p/(rho R) round trip; its float32 inputs hold p only to ~6e-8.
  rtol = 5e-5 if dtype == torch.float64 else 2e-4
  for d in DIMS:
    np.testing.assert_allclose(_np(q[d])[1:, 1:, 1:], expected[d][1:, 1:, 1:],
                               atol=5e-5, rtol=rtol, err_msg=d)


def test_intercell_diffusive_flux_zero_in_isothermal_gas():
  from swirlc_b200.equations import compressible_navier_stokes as cns
  prim = ka.isothermal_case()
  cfg = _cfg(conservative_variable_names=NAMES6)
  flux = cns._intercell_diffusive_flux(_dev(prim), cfg, _pm(cfg))
  for d in DIMS:
    assert list(flux[d]) == NAMES6
    for k, v in flux[d].items():
      np.testing.assert_allclose(_np(v)[WIN], 0.0, atol=1e-6,
                                 err_msg=f'{d} {k}')


@pytest.mark.parametrize('dim', DIMS)
def test_intercell_diffusive_flux_heat_conduction_only(dim):
  from swirlc_b200.equations import compressible_navier_stokes as cns
  prim, want, h, nu, pr = ka.heat_conduction_case(dim)
  cfg = _cfg(dx=h, dy=h, dz=h, conservative_variable_names=NAMES6,
             transport_parameters={'nu': nu, 'pr': pr})
  flux = cns._intercell_diffusive_flux(_dev(prim), cfg, _pm(cfg))
  for d in DIMS:
    for k, v in flux[d].items():
      exp = want if (d == dim and k == 'rho_e') else np.zeros_like(want)
      np.testing.assert_allclose(_np(v)[WIN], exp[WIN], atol=5e-5, rtol=5e-5,
                                 err_msg=f'{d} {k}')


def test_intercell_diffusive_flux_equals_oracle_on_a_random_state():
  from swirlc_b200.equations import compressible_navier_stokes as cns
  from tests import helpers
  cons = helpers.random_state((14, 12, 10), seed=4, dtype=np.float64)
  prim = orc.conservative_to_primitive(cons)
  prim['p'] = orc.pressure(prim, 0.0)
  tp = {'nu': 3e-2, 'pr': 0.7}
  cfg = _cfg(dx=0.3, dy=0.2, dz=0.25, transport_parameters=tp)
  ocfg = orc.make_cfg(dx=0.3, dy=0.2, dz=0.25, transport_parameters=tp)
  got = cns._intercell_diffusive_flux(_dev(prim), cfg, _pm(cfg))
  want = orc.diffusive_flux(prim, ocfg, list(orc.BASE_CONSERVATIVE))
  inner = (slice(1, -1),) * 3
  for d in DIMS:
    for k in orc.BASE_CONSERVATIVE:
      w = want[d][k][inner]
      np.testing.assert_allclose(_np(got[d][k])[inner], w, rtol=1e-11,
                                 atol=1e-11 * max(np.abs(w).max(), 1.0),
                                 err_msg=f'{d} {k}')


@pytest.mark.parametrize('dim', DIMS)
def test_fused_rhs_heat_conduction_only(dim):
  """The heat-conduction case through the fused stage (identity faces,
  viscous; periodic halos across the gradient, the given halo cells along
  it): rho_e changes by -(q[i+1] - q[i]) / h, everything else stays put."""
  from swirlc_b200.boundary import bc_types
  from swirlc_b200.equations import compressible_navier_stokes as cns
  prim, q, h, nu, pr = ka.heat_conduction_case(dim)
  cons = orc.primitive_to_conservative(
      {k: prim[k] for k in ('rho', 'u', 'v', 'w', 'e')})
  ax = orc.AXIS[dim]
  per = {0: (bc_types.BoundaryCondition.PERIODIC,),
         1: (bc_types.BoundaryCondition.PERIODIC,)}
  # An empty entry for a dim leaves its halo cells as given.
  ubc = {'cell_averages': {n: {d: (per if d != dim else {}) for d in DIMS}
                           for n in orc.BASE_CONSERVATIVE}}
  cfg = _cfg(dx=h, dy=h, dz=h, interpolation_scheme='NODE',
             numeric_flux_scheme='HLLC', include_diffusion=True,
             transport_parameters={'nu': nu, 'pr': pr}, bc=ubc)
  rhs = cns.get_rhs_fn(np.array([[[0]]]), cfg, _pm(cfg))
  out = rhs(0, _dev(cons), {})
  want = np.zeros_like(q)
  lo = [slice(None)] * 3
  hi = [slice(None)] * 3
  lo[ax] = slice(0, -1)
  hi[ax] = slice(1, None)
  want[tuple(lo)] = -(q[tuple(hi)] - q[tuple(lo)]) / h
  inner = (slice(3, -3),) * 3
  scale = np.abs(want[inner]).max()
  np.testing.assert_allclose(_np(out['rho_e'])[inner], want[inner],
                             atol=1e-6 * scale, rtol=1e-6)
  for k in ('rho', 'rho_u', 'rho_v', 'rho_w'):
    # The momentum flux p is uniform: its divergence cancels to rounding.
    np.testing.assert_allclose(_np(out[k])[inner], 0.0,
                               atol=1e-9 * 101325.0 / h, err_msg=k)


@pytest.mark.parametrize('solver', ['HLL', 'HLLC'])
@pytest.mark.parametrize('dim', DIMS)
def test_intercell_flux_standing_shock(dim, solver):
  from swirlc_b200.numerics.riemann_solver import riemann_solver
  cons, prim, expected = ka.standing_shock_case(dim)
  cfg = _cfg(numeric_flux_scheme=solver, conservative_variable_names=NAMES6)
  fn = riemann_solver.select_numeric_flux_fn(cfg)
  c, p = _dev(cons), _dev(prim)
  for fd in DIMS:
    got = fn(0, np.array([[[0]]]), c, c, p, p, {}, {}, None, fd, cfg, None)
    assert list(got) == NAMES6
    for k in NAMES6:
      np.testing.assert_allclose(_np(got[k])[WIN], expected[fd][k][WIN],
                                 rtol=1e-6, atol=1e-6, err_msg=f'{fd} {k}')


@pytest.mark.parametrize('kind', ['convective', 'total'])
def test_fused_rhs_intercell_flux_bcs(kind):
  """compressible_navier_stokes_test.py:1484-1826 through the fused
  extended stage: a uniform moving state with Dirichlet flux BCs on the x
  boundary faces (identity face values, the real HLL flux). The halo
  (left as given in the reference test) is filled here with zero-gradient
  x and periodic y, z conditions, which for the uniform state leave it as
  it is. Interior cells only (the stage writes no halo cells)."""
  from swirlc_b200.boundary import bc_types
  from swirlc_b200.equations import compressible_navier_stokes as cns
  from tests import test_oracle_rhs_mocked_cases as mc
  cons, ocfg, expected = mc.flux_bc_case(kind)
  B = bc_types.BoundaryCondition
  conv = lambda t: (None, None) if t[0] is None else (B.DIRICHLET, t[1])
  fluxes = {k: {d: {s: conv(v) for s, v in sides.items()}
                for d, sides in spec.items()}
            for k, spec in ocfg.bc['intercell_fluxes'][kind].items()}
  per = {0: (B.PERIODIC,), 1: (B.PERIODIC,)}
  cells = {k: {'x': {0: (B.NEUMANN, 0.0), 1: (B.NEUMANN, 0.0)}, 'y': per,
               'z': per} for k in NAMES6}
  cfg = _cfg(dx=1.0, dy=1.0, dz=1.0, interpolation_scheme='NODE',
             numeric_flux_scheme='HLL', conservative_variable_names=NAMES6,
             bc={'cell_averages': cells, 'intercell_fluxes': {kind: fluxes}})
  rhs = cns.get_rhs_fn(np.array([[[0]]]), cfg, _pm(cfg))
  out = rhs(0, _dev(cons), {})
  inner = (slice(3, -3),) * 3
  for k, want in expected.items():
    np.testing.assert_allclose(_np(out[k])[inner], want[inner], rtol=1e-9,
                               atol=1e-9 * max(np.abs(want).max(), 1.0),
                               err_msg=k)
