"""Seeded synthetic set-ups of the benchmark workloads.

Each builder returns (user_cfg dict for SwirlCParameters, initial conserved
state as NumPy arrays in the reference layout [nz+2h, nx+2h, ny+2h]). Halo
cells of the returned state hold the initial-condition formula evaluated on
the halo coordinates; the solver refills them before every RHS.

  sod(n)            Sod shock tube along x, n x 8 x 8, WENO5-JS + HLLC.
  kelvin_helmholtz  periodic unit cube, WENO5 + HLLC + viscous (nu, Pr).
  buoyant_bubble    gravity along z, z walls, MUSCL (van Leer) + HLL.
  riemann_batch     64 quasi-1-D Riemann problems of uneven sizes.
"""

from __future__ import annotations

from typing import Dict, Tuple

import numpy as np

from swirlc_b200.boundary import bc_types
from swirlc_b200.common import types
from swirlc_b200.physics import constant

BC = bc_types.BoundaryCondition
GAMMA = constant.GAMMA


def _cell_centres(n: int, length: float = 1.0) -> np.ndarray:
  """parameter.py:28-33: cell centres of n cells on [0, length]."""
  xx = np.linspace(0.0, length, n + 1, dtype=np.float32)
  return (xx[:-1] + 0.5 * np.diff(xx)[0]).astype(np.float32)


def _halo_coords(c: np.ndarray, hw: int) -> np.ndarray:
  d = float(c[1] - c[0])
  return np.concatenate([c[0] - d * np.arange(hw, 0, -1), c,
                         c[-1] + d * np.arange(1, hw + 1)])


def _periodic(names=types.BASE_CONSERVATIVE) -> Dict:
  return {n: {d: {0: (BC.PERIODIC,), 1: (BC.PERIODIC,)} for d in types.DIMS}
          for n in names}


def _base_cfg(nx, ny, nz, lx, ly, lz, hw) -> Dict:
  x, y, z = _cell_centres(nx, lx), _cell_centres(ny, ly), _cell_centres(nz, lz)
  return {
      'cx': 1, 'cy': 1, 'cz': 1, 'halo_width': hw,
      'nx': nx, 'ny': ny, 'nz': nz, 'core_nx': nx, 'core_ny': ny,
      'core_nz': nz, 'lx': lx, 'ly': ly, 'lz': lz,
      'x': x, 'y': y, 'z': z,
      'dx': float(np.diff(x)[0]), 'dy': float(np.diff(y)[0]),
      'dz': float(np.diff(z)[0]),
  }


def _to_cons(rho, u, v, w, p, pe=0.0, dtype=np.float32):
  e = p / ((GAMMA - 1.0) * rho) + 0.5 * (u * u + v * v + w * w) + pe
  return {'rho': rho.astype(dtype), 'rho_u': (rho * u).astype(dtype),
          'rho_v': (rho * v).astype(dtype), 'rho_w': (rho * w).astype(dtype),
          'rho_e': (rho * e).astype(dtype)}


def sod(n: int = 256, ny: int = 8, nz: int = 8, hw: int = 3,
        dtype=np.float32) -> Tuple[Dict, Dict]:
  """Sod tube on x in [0, 1]: left rho=1, p=1; right rho=0.125, p=0.1;
  periodic y, z; zero-gradient (Neumann 0, outflow) x; WENO5-JS + HLLC,
  CFL 0.5 to t = 0.2."""
  ly = lz = 0.0246
  cfg = _base_cfg(n, ny, nz, 1.0, ly, lz, hw)
  bc = _periodic()
  for name in types.BASE_CONSERVATIVE:
    bc[name]['x'] = {0: (BC.NEUMANN, 0.0), 1: (BC.NEUMANN, 0.0)}
  cfg.update({
      'interpolation_scheme': 'WENO_5', 'numeric_flux_scheme': 'HLLC',
      'include_diffusion': False, 'time_integration_scheme': 'rk3',
      'bc': {'cell_averages': bc}, 'cfl': 0.5, 't_end': 0.2, 'dt': 1e-3,
  })
  xh = _halo_coords(cfg['x'], hw)
  shape = (nz + 2 * hw, n + 2 * hw, ny + 2 * hw)
  left = (xh < 0.5)[np.newaxis, :, np.newaxis]
  rho = np.where(left, 1.0, 0.125) * np.ones(shape)
  p = np.where(left, 1.0, 0.1) * np.ones(shape)
  zero = np.zeros(shape)
  return cfg, _to_cons(rho, zero, zero, zero, p, dtype=dtype)


def kelvin_helmholtz(n: int = 256, hw: int = 3, nu: float = 1e-4,
                     pr: float = 0.7, seed: int = 0,
                     dtype=np.float32) -> Tuple[Dict, Dict]:
  """Periodic unit cube, p = 2.5: rho=2, u=+0.5 for |y-0.5|<0.25, else
  rho=1, u=-0.5; v = 0.01 sin(4 pi x); seeded uniform noise of amplitude
  1e-3 on u, v, w. WENO5 + HLLC + viscous, SSP-RK3 at CFL 0.5."""
  cfg = _base_cfg(n, n, n, 1.0, 1.0, 1.0, hw)
  cfg.update({
      'interpolation_scheme': 'WENO_5', 'numeric_flux_scheme': 'HLLC',
      'include_diffusion': True, 'time_integration_scheme': 'rk3',
      'transport_parameters': {'nu': nu, 'pr': pr},
      'bc': {'cell_averages': _periodic()}, 'cfl': 0.5, 'dt': 1e-3,
  })
  c = _halo_coords(cfg['x'], hw).astype(np.float64)
  shape = (n + 2 * hw,) * 3
  x = c[np.newaxis, :, np.newaxis]
  y = c[np.newaxis, np.newaxis, :]
  inner = np.abs(y - 0.5) < 0.25
  rho = np.where(inner, 2.0, 1.0) * np.ones(shape)
  u = np.where(inner, 0.5, -0.5) * np.ones(shape)
  v = 0.01 * np.sin(4.0 * np.pi * x) * np.ones(shape)
  w = np.zeros(shape)
  rng = np.random.default_rng(seed)
  u = u + rng.uniform(-1e-3, 1e-3, shape)
  v = v + rng.uniform(-1e-3, 1e-3, shape)
  w = w + rng.uniform(-1e-3, 1e-3, shape)
  p = 2.5 * np.ones(shape)
  return cfg, _to_cons(rho, u, v, w, p, dtype=dtype)


def buoyant_bubble(nx: int = 512, ny: int = 512, nz: int = 256, hw: int = 3,
                   lz: float = 1.0e3, dtype=np.float32) -> Tuple[Dict, Dict]:
  """Warm bubble under gravity along -z in an isothermal (T0 = 300 K)
  atmosphere p(z) = p0 exp(-G z / (R T0)), p0 = 1e5, R = 8.314/0.029 (the
  reference constant). +2 K Gaussian bubble of radius 0.2 lz centred at
  0.3 lz. Periodic x, y; z walls: rho_w Dirichlet 0, rho and rho_e
  Dirichlet to the hydrostatic profile, the rest Neumann 0. MUSCL (van Leer
  limiter) + HLL, SSP-RK3, CFL 0.2: with MUSCL (any limiter) the per-
  direction CFL 0.5 of the other set-ups is unstable on this stratified
  flow once dz is a few metres (|w| grows exponentially from round-off near
  the bubble, in float32 and float64, with or without p_ref / rho_ref), while
  0.2 stays bounded over the 50 steps."""
  lx = ly = lz * nx / nz
  cfg = _base_cfg(nx, ny, nz, lx, ly, lz, hw)
  t0, p0 = 300.0, 1.0e5
  rgas = constant.R
  zc = _halo_coords(cfg['z'], hw).astype(np.float64)
  # Potential energy on the solver's mesh (utils.mesh_local halo rule).
  zm = np.concatenate([(cfg['z'][1] - cfg['z'][0]) * np.arange(-hw, 0),
                       cfg['z'], cfg['z'][-1] + (cfg['z'][-1] - cfg['z'][-2])
                       * np.arange(1, hw + 1)]).astype(np.float64)

  def hydro(zz):
    p = p0 * np.exp(-constant.G * zz / (rgas * t0))
    rho = p / (rgas * t0)
    return rho, p

  bc = _periodic()
  rho_lo, rho_hi, rhoe_lo, rhoe_hi = [], [], [], []
  na, nb = nx + 2 * hw, ny + 2 * hw
  for l in range(hw):
    for zz, rl, el in ((zm[l], rho_lo, rhoe_lo),
                       (zm[nz + hw + l], rho_hi, rhoe_hi)):
      r, p = hydro(zz)
      rl.append(np.full((na, nb), r, dtype=np.float64))
      el.append(np.full((na, nb), p / (GAMMA - 1.0) + r * constant.G * zz,
                        dtype=np.float64))
  bc['rho']['z'] = {0: (BC.DIRICHLET, rho_lo), 1: (BC.DIRICHLET, rho_hi)}
  bc['rho_e']['z'] = {0: (BC.DIRICHLET, rhoe_lo), 1: (BC.DIRICHLET, rhoe_hi)}
  bc['rho_w']['z'] = {0: (BC.DIRICHLET, 0.0), 1: (BC.DIRICHLET, 0.0)}
  for name in ('rho_u', 'rho_v'):
    bc[name]['z'] = {0: (BC.NEUMANN, 0.0), 1: (BC.NEUMANN, 0.0)}
  cfg.update({
      'interpolation_scheme': 'MUSCL', 'muscl_limiter': 'van_leer',
      'numeric_flux_scheme': 'HLL', 'include_diffusion': False,
      'time_integration_scheme': 'rk3', 'g': {'x': 0.0, 'y': 0.0, 'z': -1.0},
      'source_functions': ['gravity'], 'bc': {'cell_averages': bc},
      'cfl': 0.2, 'dt': 1e-3,
  })
  shape = (nz + 2 * hw, nx + 2 * hw, ny + 2 * hw)
  xh = _halo_coords(cfg['x'], hw).astype(np.float64)[np.newaxis, :, np.newaxis]
  yh = _halo_coords(cfg['y'], hw).astype(np.float64)[np.newaxis, np.newaxis, :]
  zh = zc[:, np.newaxis, np.newaxis]
  rho_b, p = hydro(zh)
  r2 = ((xh - 0.5 * lx)**2 + (yh - 0.5 * ly)**2 + (zh - 0.3 * lz)**2)
  dtemp = 2.0 * np.exp(-r2 / (0.2 * lz)**2)
  temp = t0 + dtemp
  p = p * np.ones(shape)
  rho = p / (rgas * temp)
  pe = (constant.G * zm)[:, np.newaxis, np.newaxis]
  zero = np.zeros(shape)
  return cfg, _to_cons(rho, zero, zero, zero, p, pe=pe, dtype=dtype)


def buoyant_bubble_reference_states(nx: int = 512, ny: int = 512,
                                    nz: int = 256, hw: int = 3,
                                    lz: float = 1.0e3,
                                    dtype=np.float32) -> Dict[str, np.ndarray]:
  """The helper states `p_ref`, `rho_ref` of the buoyant bubble: the
  isothermal hydrostatic background (T0 = 300 K, p0 = 1e5) without the
  bubble, on the same [nz+2h, nx+2h, ny+2h] arrays, as the reference demo
  adds them (demo/buoyant_bubble/buoyant_bubble.py:321-323, 361-366). With
  them the solver reconstructs p - p_ref and applies buoyancy to
  rho - rho_ref (compressible_navier_stokes.py:299-335), which keeps the
  horizontal momentum out of the float32 rounding of the 1e5 Pa balance."""
  cfg = _base_cfg(nx, ny, nz, lz * nx / nz, lz * ny / nz, lz, hw)
  zc = _halo_coords(cfg['z'], hw).astype(np.float64)
  t0, p0 = 300.0, 1.0e5
  p = p0 * np.exp(-constant.G * zc / (constant.R * t0))
  rho = p / (constant.R * t0)
  shape = (nz + 2 * hw, nx + 2 * hw, ny + 2 * hw)
  ones = np.ones(shape)
  return {'p_ref': (p[:, np.newaxis, np.newaxis] * ones).astype(dtype),
          'rho_ref': (rho[:, np.newaxis, np.newaxis] * ones).astype(dtype)}


def riemann_batch(members: int = 64, seed: int = 0, hw: int = 3):
  """64 quasi-1-D Riemann problems: nx log-uniform in [64, 4096],
  ny = nz in {4, 8, 16, 32}; rho in [0.1, 2], p in [0.1, 10], u in [-1, 1]
  left and right; diaphragm at x = 0.5; WENO5 + HLLC; own CFL dt each."""
  rng = np.random.default_rng(seed)
  out = []
  for _ in range(members):
    nx = int(np.exp(rng.uniform(np.log(64), np.log(4096))))
    nyz = int(rng.choice([4, 8, 16, 32]))
    rl, rr = rng.uniform(0.1, 2.0, 2)
    pl, pr_ = rng.uniform(0.1, 10.0, 2)
    ul, ur = rng.uniform(-1.0, 1.0, 2)
    cfg = _base_cfg(nx, nyz, nyz, 1.0, nyz / nx, nyz / nx, hw)
    bc = _periodic()
    for name in types.BASE_CONSERVATIVE:
      bc[name]['x'] = {0: (BC.NEUMANN, 0.0), 1: (BC.NEUMANN, 0.0)}
    cfg.update({'interpolation_scheme': 'WENO_5',
                'numeric_flux_scheme': 'HLLC', 'include_diffusion': False,
                'bc': {'cell_averages': bc}, 'cfl': 0.5, 'dt': 1e-4})
    xh = _halo_coords(cfg['x'], hw)[np.newaxis, :, np.newaxis]
    shape = (nyz + 2 * hw, nx + 2 * hw, nyz + 2 * hw)
    left = xh < 0.5
    rho = np.where(left, rl, rr) * np.ones(shape)
    p = np.where(left, pl, pr_) * np.ones(shape)
    u = np.where(left, ul, ur) * np.ones(shape)
    zero = np.zeros(shape)
    out.append((cfg, _to_cons(rho, u, zero, zero, p)))
  return out
