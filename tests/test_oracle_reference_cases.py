"""CPU: the oracle against the reference's own known-answer tests.

Cases restate numerics/riemann_solver/{hll,hllc}_test.py, gradient_test.py,
interpolation_test.py, time_integration/{rk3,rk2}_test.py,
boundary/boundary_test.py and the mocked-WENO RHS tests of
equations/compressible_navier_stokes_test.py, plus golden vectors extracted
from those files (tests/golden/reference_vectors.json).
"""

import json
import os

import numpy as np
import pytest

from oracle import swirlc_oracle as orc
from tests import helpers
from tests import scenarios as sc

DIMS = ('x', 'y', 'z')
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden',
                      'reference_vectors.json')


def _f32(d):
  return {k: np.asarray(v, dtype=np.float32) for k, v in d.items()}


# ---------------------------------------------------------------- Riemann
@pytest.mark.parametrize('dim', DIMS)
def test_wave_speeds_uniform_field(dim):
  c = sc.uniform(dim)
  s_l, s_r = orc.hll_wave_speeds(_f32(c['neg']), _f32(c['pos']), dim, 0.0)
  np.testing.assert_allclose(s_l, c['s_l'], rtol=1e-6)
  np.testing.assert_allclose(s_r, c['s_r'], rtol=1e-6)
  s_l, s_m, s_r = orc.hllc_wave_speeds(_f32(c['neg']), _f32(c['pos']), dim,
                                       0.0)
  np.testing.assert_allclose(s_m, c['s_m'], rtol=1e-6)


@pytest.mark.parametrize('left_running', [True, False])
@pytest.mark.parametrize('dim', DIMS)
def test_wave_speeds_strong_shock(dim, left_running):
  c = sc.shock_speeds(dim, left_running)
  s_l, s_r = orc.hll_wave_speeds(c['neg'], c['pos'], dim, 0.0)
  np.testing.assert_allclose(s_l, c['s_l'], rtol=1e-6, atol=1e-6)
  np.testing.assert_allclose(s_r, c['s_r'], rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize('case', sorted(sc.FLUX_CASES))
@pytest.mark.parametrize('solver', ['hll', 'hllc'])
@pytest.mark.parametrize('dim', DIMS)
def test_riemann_flux_known_answers(dim, solver, case):
  c = sc.FLUX_CASES[case](dim)
  fn = orc.hll_flux if solver == 'hll' else orc.hllc_flux
  got = fn(c['cneg'], c['cpos'], c['neg'], c['pos'], {}, {}, dim,
           list(orc.BASE_CONSERVATIVE), 0.0)
  for k, want in c['flux'].items():
    scale = max(np.abs(want).max(), 1.0)
    np.testing.assert_allclose(got[k], want, rtol=1e-9, atol=1e-9 * scale,
                               err_msg=f'{solver} {case} {k}')


# ---------------------------------------------------------------- stencils
def test_golden_vectors_match_reference_gradient_tests():
  with open(GOLDEN) as f:
    gold = json.load(f)
  x = np.linspace(0, 2.0 * np.pi, 16)
  y = np.sin(x).astype(np.float32)
  h = x[1] - x[0]
  f3 = helpers.to_3d(y, 'x', (4, 16, 4))
  fwd = orc.forward_1(f3, h, 'x')[2, :, 2]
  np.testing.assert_allclose(fwd[:-1], gold['gradient_forward_1'], rtol=1e-6,
                             atol=1e-6)
  cen = orc.central_2(f3, h, 'x')[2, :, 2]
  np.testing.assert_allclose(cen[1:-1], gold['gradient_central_2'],
                             rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize('dim', DIMS)
def test_linear_interpolation(dim):
  f = np.logspace(0.0, 2.0, 16)
  f3 = helpers.to_3d(f, dim, (16, 16, 16))
  for fd in DIMS:
    got = orc.linear_interpolation(f3, fd)
    exp = np.zeros(16)
    if fd == dim:
      exp[1:] = f[:-1] + 0.5 * np.diff(f)
    else:
      exp = f
    e3 = helpers.to_3d(exp, dim, (16, 16, 16))
    np.testing.assert_allclose(got[1:, 1:, 1:], e3[1:, 1:, 1:], rtol=1e-12)


# ---------------------------------------------------------------- RK
def _stage_rhs(state):
  """rk3_test.py:40-89: 20 / 40 / -10 in stages 1 / 2 / 3 by mean rho."""
  m = float(np.mean(state['rho']))
  f = 20.0 if m < 2.0 else (40.0 if m > 2.75 else -10.0)
  return {k: np.ones_like(v) * f for k, v in state.items()}


def test_rk3_constant_and_arbitrary_rhs():
  s0 = {k: np.ones((4, 4, 4)) * (i + 1)
        for i, k in enumerate(list(orc.BASE_CONSERVATIVE) + ['rho_y'])}
  same = orc.rk3(s0, 0.1, lambda s: {k: np.zeros_like(v) for k, v in s.items()})
  for k in s0:
    np.testing.assert_array_equal(same[k], s0[k])
  out = orc.rk3(s0, 0.1, _stage_rhs)
  for k in s0:
    np.testing.assert_allclose(out[k], s0[k] + 1.0 / 3.0, rtol=1e-12)


# ---------------------------------------------------------------- halos
def test_halo_fill_matches_boundary_test_single_replica():
  """boundary_test.py:60-343 with one replica along every dim."""
  n = 16
  u0 = np.zeros((n, n, n), np.float32)
  u0[3:-3, 3:-3, 3:-3] = 6.0
  p0 = np.zeros((n, n, n), np.float32)
  p0[3:-3, 3:-3, 3:-3] = 200.0
  u_bc_z0 = [np.ones((n, n)), 2.0 * np.ones((n, n)), 3.0 * np.ones((n, n))]
  p_bc_x1 = [60.0 * np.ones((n, n)), 80.0 * np.ones((n, n)),
             120.0 * np.ones((n, n))]
  bc_u = {'x': {0: (orc.DIRICHLET, 8.0), 1: (orc.NEUMANN, 0.0)},
          'y': {0: (orc.PERIODIC,), 1: (orc.PERIODIC,)},
          'z': {0: (orc.DIRICHLET, u_bc_z0), 1: (orc.NEUMANN, 1.0)}}
  bc_p = {'x': {0: (orc.NEUMANN, 8.0), 1: (orc.DIRICHLET, p_bc_x1)},
          'y': {0: (orc.PERIODIC,), 1: (orc.PERIODIC,)},
          'z': {0: (orc.DIRICHLET, 100.0), 1: (orc.NEUMANN, 0.0)}}
  u = orc.exchange_halos(u0, bc_u, 3)
  p = orc.exchange_halos(p0, bc_p, 3)
  i = slice(3, -3)
  np.testing.assert_array_equal(u[i, :3, i], 8.0)
  np.testing.assert_array_equal(u[i, -3:, i], 6.0)
  np.testing.assert_array_equal(u[i, i, :3], 6.0)
  for l, v in enumerate((1.0, 2.0, 3.0)):
    np.testing.assert_array_equal(u[l, i, i], v)
  for l, v in enumerate((7.0, 8.0, 9.0)):
    np.testing.assert_array_equal(u[n - 3 + l, i, i], v)
  for l, v in enumerate((176.0, 184.0, 192.0)):
    np.testing.assert_array_equal(p[i, l, i], v)
  for l, v in enumerate((60.0, 80.0, 120.0)):
    np.testing.assert_array_equal(p[i, n - 3 + l, i], v)
  np.testing.assert_array_equal(p[:3, i, i], 100.0)
  np.testing.assert_array_equal(p[-3:, i, i], 200.0)


# ---------------------------------------------------------------- RHS mocks
def _plug_state(dim, v_conv, n=16):
  p = 101325.0 * np.ones(n)
  t = 300.0 * np.ones(n)
  rho = p / (orc.R * t)
  vel = [np.zeros(n), np.zeros(n), np.zeros(n)]
  vel[DIMS.index(dim)] = v_conv * np.ones(n)
  e = orc.CV * t + 0.5 * (vel[0]**2 + vel[1]**2 + vel[2]**2)
  size = (n, n, n)
  cons = {'rho': rho, 'rho_u': rho * vel[0], 'rho_v': rho * vel[1],
          'rho_w': rho * vel[2], 'rho_e': rho * e}
  return {k: helpers.to_3d(v, dim, size) for k, v in cons.items()}, rho


@pytest.mark.parametrize('dim,v_conv', [('x', 10.0), ('y', -25.0),
                                        ('z', 15.0)])
def test_rhs_plug_flow_with_identity_faces(dim, v_conv):
  """compressible_navier_stokes_test.py:976-1053 (WENO mocked to node
  values, halo update mocked away): mass and momentum are steady."""
  cons, _ = _plug_state(dim, v_conv)
  cfg = orc.make_cfg(interpolation_scheme='NODE', numeric_flux_scheme='HLL')
  out = orc.rhs(cons, cfg, apply_bc=False)
  hw = 3
  for k in orc.BASE_CONSERVATIVE:
    v = out[k][hw:-hw, hw:-hw, hw:-hw]
    scale = max(np.abs(cons[k]).max(), 1.0) / cfg.dx
    np.testing.assert_allclose(v, 0.0, atol=1e-9 * scale, err_msg=k)


def test_rhs_quiescent_gas_is_zero():
  n = 16
  cons, _ = _plug_state('x', 0.0)
  for scheme in ('WENO_5', 'WENO_3', 'MUSCL', 'NODE'):
    for flux in ('HLL', 'HLLC'):
      cfg = orc.make_cfg(interpolation_scheme=scheme, numeric_flux_scheme=flux)
      out = orc.rhs(cons, cfg)
      for k in orc.BASE_CONSERVATIVE:
        assert np.abs(out[k][3:-3, 3:-3, 3:-3]).max() < 1e-6 * 101325.0 / cfg.dx
