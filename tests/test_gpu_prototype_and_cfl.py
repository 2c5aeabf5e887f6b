"""GPU: the CUDA path against the reference prototype's own outputs, and the
device CFL time step against the oracle.

* Reconstruction (swc_reconstruct): WENO5 and the prototype's MUSCL slope
  ('minmod3') on tests/golden/prototype_vectors.json, written by the
  reference notebook's own `weno5` / `muscl` (demo/swirl_c_prototype.ipynb,
  cell 4).
* HLL (swc_riemann_flux) on the notebook's `hll` outputs (cell 11).
* CFL: swc_cfl_reduce on the notebook's printed CFL numbers (`solve`,
  cell 16), and on the benchmark set-ups (Kelvin-Helmholtz, Sod, buoyant
  bubble) against `cfl_dt_min` of the oracle; the limit fused into the
  last RK stage (dtmin_out) against the oracle on the same new state.
"""

import json
import os

import numpy as np
import pytest
import torch

from oracle import swirlc_oracle as orc

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden',
                      'prototype_vectors.json')
with open(GOLDEN) as _f:
  _DATA = json.load(_f)
AX = {'x': 1, 'y': 2, 'z': 0}
NAMES = orc.BASE_CONSERVATIVE
TORCH = {'float64': torch.float64, 'float32': torch.float32}


def _window(a, dim, lo, hi):
  idx = [slice(None)] * 3
  idx[AX[dim]] = slice(lo, hi)
  return a[tuple(idx)]


@pytest.mark.parametrize('case', _DATA['recon'], ids=[
    f"{c['scheme']}-{c['dtype']}-{c['dim']}-{c['kind']}" for c in _DATA['recon']])
def test_cuda_reconstruction_matches_prototype(case):
  from swirlc_b200.numerics import interpolation
  dt, dim = case['dtype'], case['dim']
  v = torch.tensor(np.asarray(case['v'], dtype=dt), device='cuda')
  if case['scheme'] == 'weno5':
    neg, pos = interpolation.weno(v, dim, 3)
  else:
    neg, pos = interpolation.flux_limiter(
        v, dim, interpolation.FluxLimiterType.MINMOD3)
  # swc_reconstruct sets both face values where the face's whole stencil
  # (LO cells below, RI above) is inside the array and 0 elsewhere.
  n = v.shape[AX[dim]]
  klo, khi = (3, n - 2) if case['scheme'] == 'weno5' else (2, n - 1)
  for got, key, rng in ((neg, 'neg', case['neg_range']),
                        (pos, 'pos', case['pos_range'])):
    rng = (max(rng[0], klo), min(rng[1], khi))
    g = _window(got.cpu().numpy(), dim, *rng).astype(np.float64)
    w = _window(np.asarray(case[key], dtype=dt), dim, *rng).astype(np.float64)
    if case['scheme'] == 'muscl':
      # Differences, one exact scaling, min and one fused add: bit for bit.
      np.testing.assert_array_equal(g, w, err_msg=key)
    else:
      # WENO5 with folded weights: float64 to rounding, float32 to a few ulp
      # of the fast-math reciprocals.
      tol = 1e-14 if dt == 'float64' else 3e-6
      err = np.max(np.abs(g - w) / np.maximum(np.abs(w), 1.0))
      assert err <= tol, f'{key}: {err:.3e}'


@pytest.mark.parametrize('case', _DATA['hll'],
                         ids=[f"{c['dtype']}-{c['dim']}" for c in _DATA['hll']])
def test_cuda_hll_matches_prototype(case):
  from swirlc_b200.core import parameter
  from swirlc_b200.numerics.riemann_solver import hll
  dt, dim = case['dtype'], case['dim']
  to3 = lambda a: torch.tensor(np.asarray(a, dtype=dt).reshape(-1, 1, 1),
                               device='cuda')
  cn = {k: to3(v) for k, v in case['cons_neg'].items()}
  cp = {k: to3(v) for k, v in case['cons_pos'].items()}

  def prim(c):
    p = {'rho': c['rho']}
    for k in ('u', 'v', 'w', 'e'):
      p[k] = c['rho_' + k] / c['rho']
    p['p'] = 0.4 * c['rho'] * (p['e'] - 0.5 * (p['u']**2 + p['v']**2 +
                                                p['w']**2))
    p['h'] = p['e'] + p['p'] / p['rho']
    return p

  cfg = parameter.SwirlCParameters()
  got = hll.hll_convective_flux(0, np.array([[[0]]]), cn, cp, prim(cn),
                                prim(cp), {}, {}, None, dim, cfg, None)
  scale = max(max(np.abs(np.asarray(v)).max() for v in case['flux'].values()),
              1.0)
  tol = 1e-12 if dt == 'float64' else 2e-5
  for k, want in case['flux'].items():
    g = got[k].double().cpu().numpy().reshape(-1)
    err = np.max(np.abs(g - np.asarray(want, dtype=np.float64))) / scale
    assert err <= tol, f'{k}: {err:.3e}'


def _solver(user_cfg, shape, dtype):
  from swirlc_b200 import engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  cfg = parameter.SwirlCParameters(user_cfg)
  return cfg, engine.Solver(cfg, physics_models.PhysicsModels(cfg), shape,
                            dtype)


def _cuda_cfl(solver, fields):
  out = torch.full((1,), 1e300, dtype=torch.float64, device='cuda')
  solver.cfl_reduce(fields, out)
  return float(out.item())


@pytest.mark.parametrize('case', _DATA['cfl'], ids=[
    f"{c['dtype']}-grav{int(c['gravity_z'])}" for c in _DATA['cfl']])
def test_cuda_cfl_matches_prototype(case):
  dt = case['dtype']
  hw = 3
  cons = {k: np.pad(np.asarray(v, dtype=dt), hw, mode='wrap')
          for k, v in case['cons'].items()}
  nz, nx, ny = (s - 2 * hw for s in cons['rho'].shape)
  user_cfg = {'halo_width': hw, 'nx': nx, 'ny': ny, 'nz': nz,
              'core_nx': nx, 'core_ny': ny, 'core_nz': nz,
              'x': np.asarray(case['x'], dtype=dt),
              'y': np.asarray(case['y'], dtype=dt),
              'z': np.asarray(case['z'], dtype=dt),
              'dx': case['dx'], 'dy': case['dy'], 'dz': case['dz']}
  if case['gravity_z']:
    user_cfg['g'] = {'x': 0.0, 'y': 0.0, 'z': -1.0}
  _, solver = _solver(user_cfg, cons['rho'].shape, TORCH[dt])
  fields = [torch.tensor(cons[k], device='cuda') for k in NAMES]
  got = _cuda_cfl(solver, fields)
  want = case['dt'] / max(case['cfl_xyz'])
  # With gravity the potential energy comes from the mesh coordinates,
  # which are float32 (types.DTYPE, utils.py:43-89) in both precisions.
  tol = 1e-6 if dt == 'float32' else (1e-7 if case['gravity_z'] else 1e-13)
  assert abs(got - want) <= tol * want, (got, want)


def _setups():
  from swirlc_b200 import configs
  return {
      'kh': configs.kelvin_helmholtz(n=32, nu=1e-3),
      'sod': configs.sod(),
      'bubble': configs.buoyant_bubble(nx=24, ny=20, nz=16, lz=100.0),
  }


@pytest.mark.parametrize('name', ['kh', 'sod', 'bubble'])
@pytest.mark.parametrize('dtype', [torch.float32, torch.float64])
def test_cfl_reduce_and_fused_limit_match_oracle(name, dtype):
  """swc_cfl_reduce on the initial state and the limit reduced inside the
  last RK stage (the device clock's dtmin) on the state after one step,
  both against the oracle's cfl_dt_min of the same state."""
  from swirlc_b200 import engine
  user_cfg, state = _setups()[name]
  npd = np.float32 if dtype == torch.float32 else np.float64
  tol = 1e-6 if dtype == torch.float32 else 1e-13
  cfg, solver = _solver(user_cfg, state['rho'].shape, dtype)
  ocfg = orc.make_cfg(**{k: user_cfg[k] for k in (
      'halo_width', 'dx', 'dy', 'dz', 'x', 'y', 'z', 'g') if k in user_cfg})
  fields = [torch.tensor(state[k], dtype=dtype, device='cuda') for k in NAMES]
  got = _cuda_cfl(solver, fields)
  want = orc.cfl_dt_min({k: state[k].astype(npd) for k in NAMES}, ocfg)
  assert abs(got - want) <= tol * want, (name, got, want)

  st = engine.Stepper(solver, fields, dt=cfg.dt, cfl=0.0,
                      scheme=cfg.time_integration_scheme)
  st.step(1)
  fused = float(st.clock[2].item())
  new = {k: v.cpu().numpy() for k, v in zip(NAMES, st.u)}
  want = orc.cfl_dt_min(new, ocfg)
  assert abs(fused - want) <= tol * want, (name, fused, want)
