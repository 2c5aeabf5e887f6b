"""CPU: the oracle against more of the reference's own known answers.

Restated from physics/fluid_test.py:122-145 (strain rate),
physics/diffusion_test.py:116-201 (shear stress, heat flux),
equations/compressible_navier_stokes_test.py:624-775 (standing shock),
:1979-2102 (diffusive flux: isothermal gas, heat conduction) and
physics/thermodynamics/generic_test.py:50-712 (pressure, enthalpy, sound
speed, temperature, gravitational potential, internal energy, sensible
enthalpy). The cases live in tests/known_answers.py and also drive the CUDA
path (tests/test_gpu_known_answers.py). Tolerances are the reference's
(assertAllClose defaults rtol = atol = 1e-6 unless the test states others).
"""

import numpy as np
import pytest

from oracle import swirlc_oracle as orc
from tests import known_answers as ka

DIMS = ('x', 'y', 'z')
NAMES6 = list(orc.BASE_CONSERVATIVE) + ['rho_y']
WIN = (slice(3, -2),) * 3  # [hw:-(hw-1)] with hw = 3


def test_strain_rate_taylor_green():
  states, expected, delta = ka.strain_rate_case()
  s = orc.strain_rate(states, delta)
  inner = (slice(1, -1),) * 3
  for i in range(3):
    for j in range(3):
      np.testing.assert_allclose(s[i][j][inner], expected[i][j][inner],
                                 atol=5e-2, rtol=1e-6, err_msg=f'S{i}{j}')


def test_shear_stress_taylor_green():
  states, rho_f, expected, delta, nu = ka.shear_stress_case()
  prim_f = {d: {'rho': rho_f[d]} for d in DIMS}
  tau = orc.shear_stress(states, prim_f, delta, nu)
  inner = (slice(1, -1),) * 3
  for i in range(3):
    for j in range(3):
      np.testing.assert_allclose(tau[i][j][inner], expected[i][j][inner],
                                 atol=1e-2, rtol=1e-6, err_msg=f'tau{i}{j}')


def test_single_component_heat_flux():
  prim, expected, delta, nu, pr = ka.heat_flux_case()
  q = orc.heat_flux(prim, delta, nu, pr)
  for d in DIMS:
    np.testing.assert_allclose(q[d][1:, 1:, 1:], expected[d][1:, 1:, 1:],
                               atol=5e-5, rtol=5e-5, err_msg=d)


def _cfg_default(h=None):
  cfg = orc.make_cfg()
  if h is not None:
    cfg.dx = cfg.dy = cfg.dz = h
  return cfg


def test_diffusive_flux_zero_in_isothermal_gas():
  prim = ka.isothermal_case()
  flux = orc.diffusive_flux(prim, _cfg_default(), NAMES6)
  for d in DIMS:
    assert list(flux[d]) == NAMES6
    for k, v in flux[d].items():
      np.testing.assert_allclose(v[WIN], 0.0, atol=1e-6, err_msg=f'{d} {k}')


@pytest.mark.parametrize('dim', DIMS)
def test_diffusive_flux_heat_conduction_only(dim):
  prim, want, h, nu, pr = ka.heat_conduction_case(dim)
  cfg = _cfg_default(h)
  cfg.transport_parameters = {'nu': nu, 'pr': pr}
  flux = orc.diffusive_flux(prim, cfg, NAMES6)
  for d in DIMS:
    for k, v in flux[d].items():
      exp = want if (d == dim and k == 'rho_e') else np.zeros_like(v)
      np.testing.assert_allclose(v[WIN], exp[WIN], atol=5e-5, rtol=5e-5,
                                 err_msg=f'{d} {k}')


@pytest.mark.parametrize('solver', ['hll', 'hllc'])
@pytest.mark.parametrize('dim', DIMS)
def test_intercell_flux_standing_shock(dim, solver):
  """Equal face states on both sides: the Riemann flux is the physical
  flux, continuous across the Mach-6 shock (Rankine-Hugoniot)."""
  cons, prim, expected = ka.standing_shock_case(dim)
  fn = orc.hll_flux if solver == 'hll' else orc.hllc_flux
  for fd in DIMS:
    got = fn(cons, cons, prim, prim, {}, {}, fd, NAMES6, 0.0)
    for k in NAMES6:
      np.testing.assert_allclose(got[k][WIN], expected[fd][k][WIN],
                                 rtol=1e-6, atol=1e-6, err_msg=f'{fd} {k}')


# ------------------------------------------------- thermodynamics (generic)
def _thermo_cfg(g=None):
  xx = np.linspace(0.0, 1800.0, 10)
  cfg = orc.make_cfg(x=xx, y=xx, z=xx, nx=10, ny=10, nz=10,
                     dx=200.0, dy=200.0, dz=200.0)
  cfg.g = dict(g or {'x': 0.0, 'y': 0.0, 'z': 0.0})
  return cfg


SIZE16 = [16, 16, 16]
LINE = dict(u=np.linspace(-3.0, 12.0, 16), v=np.linspace(6.0, -24.0, 16),
            w=np.linspace(-9.0, 36.0, 16))
# The mesh of the 10-point coordinates with the halo rule (utils.py:58-73).
ZH = np.linspace(-600.0, 2400.0, 16)


@pytest.mark.parametrize('dim', DIMS)
def test_pressure_from_total_energy(dim):
  """generic_test.py:49-83 (constant potential temperature 300 K)."""
  cfg = _thermo_cfg({**{'x': 0.0, 'y': 0.0, 'z': 0.0}, dim: -1.0})
  theta = 300.0
  p = orc.P_0 * (1.0 - orc.G * ZH / orc.CP / theta)**(1.0 / orc.KAPPA)
  t = theta * (p / orc.P_0)**orc.KAPPA
  rho = p / orc.R / t
  e = 0.5 * (LINE['u']**2 + LINE['v']**2 + LINE['w']**2) + orc.G * ZH + \
      orc.CV * t
  st = {'rho': ka.to_3d(rho, dim, SIZE16), 'e': ka.to_3d(e, dim, SIZE16)}
  st.update({k: ka.to_3d(v, dim, SIZE16) for k, v in LINE.items()})
  pe = orc.potential_energy(cfg, st['rho'].shape, np.float64)
  np.testing.assert_allclose(orc.pressure(st, pe), ka.to_3d(p, dim, SIZE16),
                             rtol=1e-6, atol=1e-6)


def _ke_t():
  t = np.linspace(250.0, 3000.0, 16)
  ke = 0.5 * (LINE['u']**2 + LINE['v']**2 + LINE['w']**2)
  return ke, t


@pytest.mark.parametrize('dim', DIMS)
def test_total_enthalpy_and_sound_speeds(dim):
  """generic_test.py:84-240: total enthalpy from e; sound speed from e, from
  h and from (p, rho); the error for an unknown option."""
  cfg = _thermo_cfg({**{'x': 0.0, 'y': 0.0, 'z': 0.0}, dim: -1.0})
  ke, t = _ke_t()
  rho = np.logspace(-1.0, 2.0, 16)
  e = ke + orc.G * ZH + orc.CV * t
  st = {'rho': ka.to_3d(rho, dim, SIZE16), 'e': ka.to_3d(e, dim, SIZE16)}
  st.update({k: ka.to_3d(v, dim, SIZE16) for k, v in LINE.items()})
  pe = orc.potential_energy(cfg, st['rho'].shape, np.float64)
  np.testing.assert_allclose(
      orc.total_enthalpy(st, pe),
      ka.to_3d(orc.CP * t + ke + orc.G * ZH, dim, SIZE16), rtol=1e-6, atol=1e-6)
  c = ka.to_3d(np.sqrt(orc.GAMMA * orc.R * t), dim, SIZE16)
  np.testing.assert_allclose(orc.sound_speed(st, pe, 'e'), c, rtol=1e-6,
                             atol=1e-6)
  sh = {k: v for k, v in st.items() if k != 'e'}
  sh['h'] = ka.to_3d(ke + orc.G * ZH + orc.CP * t, dim, SIZE16)
  np.testing.assert_allclose(orc.sound_speed(sh, pe, 'h'), c, rtol=1e-6,
                             atol=1e-6)
  p = np.logspace(3.0, 6.0, 16)
  sp = {'rho': ka.to_3d(p / (orc.R * t), dim, SIZE16),
        'p': ka.to_3d(p, dim, SIZE16)}
  np.testing.assert_allclose(orc.sound_speed(sp, pe, 'p_rho'), c, rtol=1e-6,
                             atol=1e-6)
  with pytest.raises(ValueError, match='not a valid option for sound speed'):
    orc.sound_speed(sp, pe, 'bad_option')


@pytest.mark.parametrize('dim', DIMS)
def test_temperature_from_eos(dim):
  """generic_test.py:294-320."""
  p = np.logspace(3.0, 6.0, 16)
  rho = np.logspace(-1.0, 2.0, 16)
  st = {'p': ka.to_3d(p, dim, SIZE16), 'rho': ka.to_3d(rho, dim, SIZE16)}
  np.testing.assert_allclose(orc.temperature_eos(st),
                             ka.to_3d(p / (rho * orc.R), dim, SIZE16),
                             rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize('gravity_dim', ['x', 'y', 'z', 'w'])
def test_gravitational_potential_one_replica(gravity_dim):
  """generic_test.py:421-451 ('w': no gravity)."""
  g = {'x': 0.0, 'y': 0.0, 'z': 0.0}
  if gravity_dim != 'w':
    g[gravity_dim] = -1.0
  cfg = _thermo_cfg(g)
  pe = orc.potential_energy(cfg, (16, 16, 16), np.float64)
  dim = gravity_dim if gravity_dim != 'w' else 'z'
  gg = orc.G if gravity_dim != 'w' else 0.0
  np.testing.assert_allclose(pe, ka.to_3d(ZH * gg, dim, SIZE16), rtol=1e-6,
                             atol=1e-6)


THETA = tuple(np.pi * np.linspace(0.0, 1.0, 6)[:-1])
PHI = tuple(np.pi * np.linspace(-1.0, 1.0, 8)[1:])
ANGLES = [(t, p) for t in THETA for p in PHI]


def _angled(theta, phi):
  g = {'x': np.sin(phi) * np.cos(theta), 'y': np.sin(phi) * np.sin(theta),
       'z': np.cos(phi)}
  pe = -orc.G * (ka.to_3d(ZH * g['x'], 'x', SIZE16) +
                 ka.to_3d(ZH * g['y'], 'y', SIZE16) +
                 ka.to_3d(ZH * g['z'], 'z', SIZE16))
  return _thermo_cfg(g), pe


@pytest.mark.parametrize('theta,phi', ANGLES)
def test_gravitational_potential_arbitrary_angle(theta, phi):
  """generic_test.py:453-479 (atol 10, rtol SMALL)."""
  cfg, want = _angled(theta, phi)
  pe = orc.potential_energy(cfg, (16, 16, 16), np.float64)
  np.testing.assert_allclose(pe, want, atol=10.0, rtol=orc.SMALL)


@pytest.mark.parametrize('dim', DIMS)
@pytest.mark.parametrize('theta,phi', ANGLES)
def test_internal_energy_and_sensible_enthalpy_with_gravity(theta, phi, dim):
  """generic_test.py:620-710: e_int = e - ke - pe and h_s = h - ke - pe with
  misaligned gravity (atol 10, rtol SMALL)."""
  cfg, pe_want = _angled(theta, phi)
  ke, t = _ke_t()
  pe = orc.potential_energy(cfg, (16, 16, 16), np.float64)
  st = {k: ka.to_3d(v, dim, SIZE16) for k, v in LINE.items()}
  st['e'] = pe_want + ka.to_3d(ke + orc.CV * t, dim, SIZE16)
  np.testing.assert_allclose(orc.internal_energy(st, pe),
                             ka.to_3d(orc.CV * t, dim, SIZE16), atol=10.0,
                             rtol=orc.SMALL)
  st['h'] = pe_want + ka.to_3d(ke + orc.CP * t, dim, SIZE16)
  np.testing.assert_allclose(orc.sensible_enthalpy(st, pe),
                             ka.to_3d(orc.CP * t, dim, SIZE16), atol=10.0,
                             rtol=orc.SMALL)
