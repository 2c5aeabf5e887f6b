"""Known-answer cases of the reference's own test files, restated in NumPy.

Each generator rebuilds the inputs and the expected values of one reference
test (cited file:line), in the reference layout [nz, nx, ny], so that the
same case checks the oracle on CPU (tests/test_oracle_known_answers.py) and
the CUDA path on a GPU (tests/test_gpu_known_answers.py).
"""

import numpy as np

from oracle import swirlc_oracle as orc

DIMS = ('x', 'y', 'z')


def to_3d(f, dim, size):
  """common/testing_utils.py:23-62: a 1-D profile along `dim`, tiled."""
  f = np.asarray(f, dtype=np.float64)
  nx, ny, nz = size
  if dim == 'x':
    return np.tile(f[np.newaxis, :, np.newaxis], (nz, 1, ny))
  if dim == 'y':
    return np.tile(f[np.newaxis, np.newaxis, :], (nz, nx, 1))
  return np.tile(f[:, np.newaxis, np.newaxis], (1, nx, ny))


def tgv_fine(nx=16, ny=16, nz=16):
  """Taylor-Green fields on the doubled grid of the diffusion and fluid
  tests (diffusion_test.py:35-57, fluid_test.py:55-70): x-y-z arrays and
  the spacing h per dim."""
  n_tot = [2 * n for n in (nx, ny, nz)]
  h = [np.pi / (n - 1) for n in (nx, ny, nz)]
  x, y, z = [hi * np.arange(n) for hi, n in zip(h, n_tot)]
  xx, yy, zz = np.meshgrid(x, y, z, indexing='ij')
  f = {
      'u': np.cos(xx) * np.sin(yy) * np.sin(zz),
      'v': np.sin(xx) * np.cos(yy) * np.sin(zz),
      'w': np.sin(xx) * np.sin(yy) * np.cos(zz),
      'rho': 0.5 * (np.sin(xx) * np.sin(yy) * np.sin(yy) + 2.0),
      's_12': np.cos(xx) * np.cos(yy) * np.sin(zz),
      's_13': np.cos(xx) * np.sin(yy) * np.cos(zz),
      's_23': np.sin(xx) * np.cos(yy) * np.cos(zz),
      's_kk': np.zeros(n_tot),
  }
  return f, h


def _zxy(a):
  return np.ascontiguousarray(np.transpose(a, (2, 0, 1)))


_S_NAMES = [['s_kk', 's_12', 's_13'], ['s_12', 's_kk', 's_23'],
            ['s_13', 's_23', 's_kk']]


def strain_rate_case():
  """fluid_test.py:55-145: cell values on the even nodes, S_ij expected on
  the j faces (index i holds face i-1/2), compared on [1:-1]^3 with atol
  5e-2."""
  f, h = tgv_fine()
  nx = ny = nz = 16
  states = {k: _zxy(f[k][::2, ::2, ::2]) for k in ('u', 'v', 'w', 'rho')}

  def face(s_full, dim):
    s_face = np.zeros((nx, ny, nz))
    if dim == 'x':
      s_face[1:, :, :] = s_full[1:-1:2, ::2, ::2]
    elif dim == 'y':
      s_face[:, 1:, :] = s_full[::2, 1:-1:2, ::2]
    else:
      s_face[:, :, 1:] = s_full[::2, ::2, 1:-1:2]
    return _zxy(s_face)

  s = [[face(f[_S_NAMES[i][j]], DIMS[j]) for j in range(3)] for i in range(3)]
  delta = {d: 2.0 * hi for d, hi in zip(DIMS, h)}
  return states, s, delta


def shear_stress_case():
  """diffusion_test.py:35-146: cell values on the odd nodes, face densities
  from the fine grid, tau_ij = 0.2 rho_j S_ij (nu = 0.1), compared on
  [1:-1]^3 with atol 1e-2."""
  f, h = tgv_fine()
  states = {k: _zxy(f[k][1::2, 1::2, 1::2]) for k in ('u', 'v', 'w', 'rho')}
  rho = f['rho']
  rho_f = {'x': _zxy(rho[::2, 1::2, 1::2]), 'y': _zxy(rho[1::2, ::2, 1::2]),
           'z': _zxy(rho[1::2, 1::2, ::2])}

  def face(s_full, dim):
    if dim == 'x':
      return _zxy(s_full[::2, 1::2, 1::2])
    if dim == 'y':
      return _zxy(s_full[1::2, ::2, 1::2])
    return _zxy(s_full[1::2, 1::2, ::2])

  tau = [[0.2 * rho_f[DIMS[j]] * face(f[_S_NAMES[i][j]], DIMS[j])
          for j in range(3)] for i in range(3)]
  delta = {d: 2.0 * hi for d, hi in zip(DIMS, h)}
  return states, rho_f, tau, delta, 0.1


def heat_flux_case(seed=0):
  """diffusion_test.py:148-201: random T in [300, 500], rho in [0.5, 1.5],
  nu = 2e-4, pr = 0.7, dx, dy, dz = 1, 2, 3 (size [16, 18, 12] in
  [nz, nx, ny]); expected -kappa_f dT/dh, compared on [1:, 1:, 1:] with
  atol = rtol = 5e-5."""
  rng = np.random.default_rng(seed)
  size = [16, 18, 12]
  t = rng.uniform(300.0, 500.0, size)
  rho = rng.uniform(0.5, 1.5, size)
  p = rho * orc.R * t
  nu, pr = 2.0e-4, 0.7
  delta = {'x': 1.0, 'y': 2.0, 'z': 3.0}
  kappa = nu / pr * rho * orc.CP
  kf = {d: np.zeros(size) for d in DIMS}
  kf['x'][:, 1:, :] = kappa[:, :-1, :] + 0.5 * np.diff(kappa, axis=1)
  kf['y'][:, :, 1:] = kappa[:, :, :-1] + 0.5 * np.diff(kappa, axis=2)
  kf['z'][1:, :, :] = kappa[:-1, :, :] + 0.5 * np.diff(kappa, axis=0)
  dtdh = {d: np.zeros(size) for d in DIMS}
  dtdh['x'][:, 1:, :] = np.diff(t, axis=1) / delta['x']
  dtdh['y'][:, :, 1:] = np.diff(t, axis=2) / delta['y']
  dtdh['z'][1:, :, :] = np.diff(t, axis=0) / delta['z']
  expected = {d: -kf[d] * dtdh[d] for d in DIMS}
  return {'rho': rho, 'p': p}, expected, delta, nu, pr


def isothermal_case():
  """compressible_navier_stokes_test.py:1979-2027: uniform velocity and
  temperature; every diffusive flux is 0 on [hw:-(hw-1)]^3."""
  nx = 16
  size = [nx] * 3
  p = 101325.0 * np.ones(nx)
  t = 500.0 * np.ones(nx)
  rho = p / (orc.R * t)
  u, v, w = 10.0 * np.ones(nx), -20.0 * np.ones(nx), 25.0 * np.ones(nx)
  e = orc.CV * t + 0.5 * (u**2 + v**2 + w**2)
  prim = {'rho': rho, 'u': u, 'v': v, 'w': w, 'e': e, 'p': p,
          'y': 0.5 * np.ones(nx)}
  return {k: to_3d(val, 'x', size) for k, val in prim.items()}


def heat_conduction_case(dim):
  """compressible_navier_stokes_test.py:2029-2102: stationary gas, T linear
  from 400 to 500 along `dim`, h = 0.5; the only non-zero diffusive flux
  is rho_e across `dim` faces: -kappa_f dT/dh (face i-1/2 at index i);
  compared on [hw:-(hw-1)]^3 with atol = rtol = 5e-5. Default transport
  parameters nu = 1e-4, pr = 0.7."""
  nx = 16
  size = [nx] * 3
  h = 0.5
  z = np.zeros(nx)
  p = 101325.0 * np.ones(nx)
  t = 400.0 + np.linspace(0.0, 100.0, nx)
  rho = p / (orc.R * t)
  e = orc.CV * t
  prim = {'rho': rho, 'u': z, 'v': z, 'w': z, 'e': e, 'p': p,
          'y': 0.5 * np.ones(nx)}
  nu, pr = 1.0e-4, 0.7
  kappa = nu / pr * rho * orc.CP
  kf = kappa[:-1] + 0.5 * np.diff(kappa)
  flux = np.zeros(nx)
  flux[1:] = -kf * np.diff(t) / h
  return ({k: to_3d(val, dim, size) for k, val in prim.items()},
          to_3d(flux, dim, size), h, nu, pr)


def normal_shock_relations(m, gamma=orc.GAMMA):
  """Pressure, density and temperature ratios across a normal shock of
  Mach m (compressible_navier_stokes_test.py:286-295)."""
  p1_p0 = (2.0 * gamma * m**2 - (gamma - 1.0)) / (gamma + 1.0)
  r1_r0 = (gamma + 1.0) * m**2 / ((gamma - 1.0) * m**2 + 2.0)
  return p1_p0, r1_r0, p1_p0 / r1_r0


def standing_shock_case(dim):
  """compressible_navier_stokes_test.py:624-775: a Mach-6 standing shock
  along `dim` (16 cells, jump at 8), the same state on both sides of every
  face. Expected convective flux across `dim` faces: rho0 u0, rho0 u0^2 +
  p0 (aligned momentum), rho0 h0 u0, rho0 y u0; across the other faces
  only the pressure p in the aligned momentum. Compared on
  [hw:-(hw-1)]^3."""
  nx = 16
  size = [nx] * 3
  m, t0, p0 = 6.0, 300.0, 101325.0
  rho0 = p0 / (orc.R * t0)
  u0 = m * np.sqrt(orc.GAMMA * orc.R * t0)
  h0 = orc.CP * t0 + 0.5 * u0**2
  _, r1_r0, t1_t0 = normal_shock_relations(m)

  def step(a, b):
    f = np.zeros(nx)
    f[:nx // 2] = a
    f[nx // 2:] = b
    return f

  rho = step(rho0, r1_r0 * rho0)
  t = step(t0, t1_t0 * t0)
  p = rho * orc.R * t
  vel = {'u': np.zeros(nx), 'v': np.zeros(nx), 'w': np.zeros(nx)}
  vel['uvw'[DIMS.index(dim)]] = step(u0, u0 / r1_r0)
  ke = 0.5 * (vel['u']**2 + vel['v']**2 + vel['w']**2)
  e = orc.CV * t + ke
  h = orc.CP * t + ke
  y = 0.5 * np.ones(nx)
  prim = {'rho': rho, 'u': vel['u'], 'v': vel['v'], 'w': vel['w'], 'e': e,
          'y': y, 'h': h, 'p': p}
  cons = {'rho': rho, 'rho_u': rho * vel['u'], 'rho_v': rho * vel['v'],
          'rho_w': rho * vel['w'], 'rho_e': rho * e, 'rho_y': rho * y}
  prim = {k: to_3d(v, dim, size) for k, v in prim.items()}
  cons = {k: to_3d(v, dim, size) for k, v in cons.items()}
  expected = {}
  names = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e', 'rho_y')
  for fd in DIMS:
    mom = 'rho_' + 'uvw'[DIMS.index(fd)]
    if fd == dim:
      ex = {'rho': rho0 * u0 * np.ones(nx), 'rho_u': np.zeros(nx),
            'rho_v': np.zeros(nx), 'rho_w': np.zeros(nx),
            'rho_e': rho0 * h0 * u0 * np.ones(nx),
            'rho_y': rho0 * y * u0}
      ex[mom] = ex[mom] + (rho0 * u0**2 + p0)
    else:
      ex = {k: np.zeros(nx) for k in names}
      ex[mom] = ex[mom] + p
    expected[fd] = {k: to_3d(v, dim, size) for k, v in ex.items()}
  return cons, prim, expected
