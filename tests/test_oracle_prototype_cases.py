"""CPU: the oracle against the reference's own runnable NumPy prototype.

tests/golden/prototype_vectors.json holds outputs of the prototype notebook's
own functions (demo/swirl_c_prototype.ipynb: `weno5` and `muscl` of cell 4,
`rk3` of cell 5, `hll` of cell 11 and the CFL numbers printed by `solve`,
cell 16), executed on seeded inputs by tests/golden/make_prototype_fixtures.py
and re-indexed to the production convention (index i holds face i-1/2,
layout [nz, nx, ny]). These pin the oracle's WENO5 (`weno(k=3)`), the
prototype MUSCL slope (`muscl(limiter='minmod3')`), the HLL flux, RK3 and
`cfl_dt_min`.
"""

import json
import os

import numpy as np
import pytest

from oracle import swirlc_oracle as orc

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden',
                      'prototype_vectors.json')
AX = {'x': 1, 'y': 2, 'z': 0}
# Relative tolerances per dtype for HLL, RK3 and CFL, whose oracle forms
# differ from the prototype's in operation order (reciprocal-multiply vs
# division, Python-float vs dtype constants).
RTOL = {'float64': 1e-13, 'float32': 2e-6}


def _load():
  with open(GOLDEN) as f:
    return json.load(f)


_DATA = _load()


def _arr(x, dt):
  return np.asarray(x, dtype=dt)


def _window(a, dim, lo, hi):
  idx = [slice(None)] * 3
  idx[AX[dim]] = slice(lo, hi)
  return a[tuple(idx)]


def _close(got, want, dt, what):
  got = np.asarray(got, dtype=np.float64)
  want = np.asarray(want, dtype=np.float64)
  scale = np.maximum(np.abs(want), 1.0 if dt == 'float32' else 1e-300)
  err = np.max(np.abs(got - want) / scale) if want.size else 0.0
  assert err <= RTOL[dt], f'{what}: max rel err {err:.3e}'


def _recon_ids():
  return [f"{c['scheme']}-{c['dtype']}-{c['dim']}-{c['kind']}"
          for c in _DATA['recon']]


@pytest.mark.parametrize('case', _DATA['recon'], ids=_recon_ids())
def test_reconstruction_matches_prototype(case):
  dt, dim = case['dtype'], case['dim']
  v = _arr(case['v'], dt)
  if case['scheme'] == 'weno5':
    neg, pos = orc.weno(v, dim, k=3)
  else:
    neg, pos = orc.muscl(v, dim, limiter='minmod3')
  assert neg.dtype == np.dtype(dt) and pos.dtype == np.dtype(dt)
  # Same formulas in the same operation order: equal to the bit.
  for got, key, rng in ((neg, 'neg', case['neg_range']),
                        (pos, 'pos', case['pos_range'])):
    want = _arr(case[key], dt)
    np.testing.assert_array_equal(_window(got, dim, *rng),
                                  _window(want, dim, *rng),
                                  err_msg=f'{case["scheme"]} {key}')


@pytest.mark.parametrize('case', _DATA['hll'],
                         ids=[f"{c['dtype']}-{c['dim']}" for c in _DATA['hll']])
def test_hll_flux_matches_prototype(case):
  dt, dim = case['dtype'], case['dim']
  cn = {k: _arr(v, dt) for k, v in case['cons_neg'].items()}
  cp = {k: _arr(v, dt) for k, v in case['cons_pos'].items()}
  pn = orc.conservative_to_primitive(cn)
  pp = orc.conservative_to_primitive(cp)
  zero = np.zeros_like(cn['rho'])
  for prim in (pn, pp):
    prim['p'] = orc.pressure(prim, zero)
    prim['h'] = orc.total_enthalpy(prim, zero)
  got = orc.hll_flux(cn, cp, pn, pp, {}, {}, dim,
                     list(orc.BASE_CONSERVATIVE), zero)
  for k, want in case['flux'].items():
    want = _arr(want, dt)
    # Fluxes are O(1); compare relative to the largest flux component, since
    # t3 * (U_R - U_L) cancels to rounding for the equal states.
    scale = max(np.abs(want).max(), 1.0)
    err = np.max(np.abs(got[k].astype(np.float64) - want)) / scale
    assert err <= 4 * RTOL[dt], f'{k}: {err:.3e}'


@pytest.mark.parametrize('case', _DATA['rk3'],
                         ids=[c['dtype'] for c in _DATA['rk3']])
def test_rk3_matches_prototype(case):
  dt = case['dtype']
  a, b = _arr(case['a'], dt), _arr(case['b'], dt)
  s0 = {k: _arr(v, dt) for k, v in case['state0'].items()}
  got = orc.rk3(s0, type(a[0])(case['dt']), lambda s: {k: a * v + b
                                                       for k, v in s.items()})
  for k, want in case['state1'].items():
    _close(got[k], _arr(want, dt), dt, f'rk3 {k}')


def _cfl_cfg(case):
  hw = 3
  nz, nx, ny = np.asarray(case['cons']['rho']).shape
  dt = case['dtype']
  cfg = orc.make_cfg(halo_width=hw, nx=nx, ny=ny, nz=nz,
                     x=_arr(case['x'], dt), y=_arr(case['y'], dt),
                     z=_arr(case['z'], dt), dx=case['dx'], dy=case['dy'],
                     dz=case['dz'])
  if case['gravity_z']:
    cfg.g = {'x': 0.0, 'y': 0.0, 'z': -1.0}
  return cfg


def _with_halo(a, hw):
  return np.pad(a, hw, mode='wrap')


@pytest.mark.parametrize('case', _DATA['cfl'],
                         ids=[f"{c['dtype']}-grav{int(c['gravity_z'])}"
                              for c in _DATA['cfl']])
def test_cfl_dt_matches_prototype(case):
  """dt / max_d CFL_d of the prototype equals the oracle's dt limit.

  The prototype prints CFL_d = max(|u_d| + c) dt / delta_d; the largest dt
  with every CFL_d <= 1 is min_d delta_d / max(|u_d| + c), which is what
  `cfl_dt_min` returns (min over cells of delta_d / (|u_d| + c)).
  """
  dt = case['dtype']
  cfg = _cfl_cfg(case)
  hw = cfg.halo_width
  cons = {k: _with_halo(_arr(v, dt), hw) for k, v in case['cons'].items()}
  got = orc.cfl_dt_min(cons, cfg)
  want = case['dt'] / max(case['cfl_xyz'])
  tol = 1e-12 if dt == 'float64' else 2e-6
  assert abs(got - want) <= tol * want, (got, want)
