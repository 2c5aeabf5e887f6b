"""CPU: the oracle's RHS against the reference's RHS tests that patch parts of
the solver (equations/compressible_navier_stokes_test.py:1063-1977,
2208-2290).

The reference patches swirl_lm's weno (node values), its own
update_conservative_cell_averages (halo left as given),
_intercell_convective_flux, _intercell_diffusive_flux, gradient.forward_1
and the physics models' source function; the oracle's `rhs` takes the same
replacements as keyword hooks, so these tests pin the oracle's BC plumbing
(cell averages, face values, convective and total flux BCs), divergence and
source handling. The flux-BC cases, which patch nothing but the
interpolation and the halo fill, also run through the CUDA path
(tests/test_gpu_known_answers.py). Set-up as the reference's
NavierStokesTest: WENO_3 (patched to node values), HLL, no diffusion, the
base conserved variables plus rho_y; 16^3 arrays with halo width 3.
"""

import numpy as np
import pytest

from oracle import swirlc_oracle as orc
from tests import known_answers as ka

NX = 16
SIZE = [NX] * 3
NAMES = list(orc.BASE_CONSERVATIVE) + ['rho_y']
SMALL = orc.SMALL
D, N, P = orc.DIRICHLET, orc.NEUMANN, orc.PERIODIC
NONE_SIDE = {0: (None, None), 1: (None, None)}


def _cfg(**kw):
  base = dict(interpolation_scheme='WENO_3', numeric_flux_scheme='HLL',
              include_diffusion=False, conservative_variable_names=NAMES,
              primitive_variable_names=list(orc.BASE_PRIMITIVES) + ['y'],
              bc={})
  base.update(kw)
  return orc.make_cfg(**base)


def _node(v, dim):
  return v, v


def _flux_return_conservative(c_neg, c_pos, p_neg, p_pos):
  """_mock_intercell_flux_function_return_conservative (:135-164)."""
  return {d: dict(c_neg['x']) for d in orc.DIMS}


def _flux_return_zeros(c_neg, c_pos, p_neg, p_pos):
  """_mock_intercell_flux_function_return_zeros (:167-197)."""
  return {d: {k: np.zeros_like(v) for k, v in c_neg['x'].items()}
          for d in orc.DIMS}


def _profiles(zfn):
  """Flux profiles of the arbitrary-flux mocks (:70-132, :200-244): sin
  along x and y, `zfn` along z, times 1..6 per variable."""
  xv = np.sin(np.linspace(0.0, 1.0, 16) * 2.0 * np.pi)
  yv = np.sin(np.linspace(0.0, 1.0, 16) * 2.0 * np.pi + np.pi / 3.0)
  zv = zfn(np.linspace(0.0, 1.0, 16))
  fac = dict(zip(NAMES, (1.0, 2.0, 3.0, 4.0, 5.0, 6.0)))
  return {d: {k: ka.to_3d(vec * f, d, SIZE) for k, f in fac.items()}
          for d, vec in (('x', xv), ('y', yv), ('z', zv))}, (xv, yv, zv)


def _forward_diff(vec):
  out = np.zeros(NX)
  out[:-1] = -np.diff(vec)
  return out


def _kh_like_state(y_profile):
  u, v, w = 10.0 * np.ones(NX), -25.0 * np.ones(NX), 15.0 * np.ones(NX)
  p = 101325.0 * np.ones(NX)
  t = 300.0 * np.ones(NX)
  rho = p / (orc.R * t)
  e = orc.CV * t + 0.5 * (u**2 + v**2 + w**2)
  return {'rho': ka.to_3d(rho, 'x', SIZE),
          'rho_u': ka.to_3d(rho * u, 'x', SIZE),
          'rho_v': ka.to_3d(rho * v, 'x', SIZE),
          'rho_w': ka.to_3d(rho * w, 'x', SIZE),
          'rho_e': ka.to_3d(rho * e, 'x', SIZE),
          'rho_y': ka.to_3d(rho * y_profile, 'x', SIZE)}


def _check(got, expected, window, rtol=2.0 * SMALL):
  assert list(got) == NAMES
  for k, want in expected.items():
    np.testing.assert_allclose(got[k][window], want[window], rtol=rtol,
                               atol=1e-9 * max(np.abs(want).max(), 1.0),
                               err_msg=k)


INTERIOR = (slice(3, -3),) * 3
WIN_LO = (slice(2, -3),) * 3  # [hw-1:-hw]


def test_specified_intercell_convective_flux():
  """:1063-1147 (patched convective flux, halo left as given)."""
  flux, (xv, yv, zv) = _profiles(lambda t: t**2.0)
  cfg = _cfg(dx=1.0, dy=1.0, dz=1.0)
  cons = _kh_like_state(np.linspace(0.0, 1.0, NX))
  got = orc.rhs(cons, cfg, interp_fn=_node, apply_bc=False,
                conv_flux_fn=lambda *a: flux)
  m = (ka.to_3d(_forward_diff(xv), 'x', SIZE) +
       ka.to_3d(_forward_diff(yv), 'y', SIZE) +
       ka.to_3d(_forward_diff(zv), 'z', SIZE))
  _check(got, {k: m * f for k, f in zip(NAMES, (1, 2, 3, 4, 5, 6))},
         INTERIOR)


def _uniform(val=0.5):
  return {k: ka.to_3d(val * np.ones(NX), 'x', SIZE) for k in NAMES}


def _x_only(lo, hi):
  return {'x': {0: (D, lo), 1: (D, hi)}, 'y': {0: (P,), 1: (P,)},
          'z': {0: (P,), 1: (P,)}}


def test_bc_updates_cell_averages_x_only():
  """:1149-1314: Dirichlet 1 / 2 cell averages in x, patched flux returning
  the (node) face values: the x divergence of the filled field."""
  cfg = _cfg()
  cfg.bc = {'cell_averages': {k: _x_only(1.0, 2.0) for k in NAMES}}
  got = orc.rhs(_uniform(), cfg, interp_fn=_node,
                conv_flux_fn=_flux_return_conservative)
  vec = 0.5 * np.ones(NX)
  vec[:3] = 1.0
  vec[-3:] = 2.0
  rhs = ka.to_3d(_forward_diff(vec) / cfg.dx, 'x', SIZE)
  _check(got, {k: rhs for k in NAMES}, WIN_LO)


def test_bc_updates_cell_faces_x_only():
  """:1316-1482: Dirichlet 1 / 2 face values in x (density included), the
  flux patched to return the face values: only the two boundary faces
  (indices 3 and 13) change."""
  cfg = _cfg(dx=1.0, dy=1.0, dz=1.0)
  faces = {k: {'x': {0: (D, 1.0), 1: (D, 2.0)}, 'y': dict(NONE_SIDE),
               'z': dict(NONE_SIDE)} for k in NAMES}
  cfg.bc = {'cell_faces': faces}
  got = orc.rhs(_uniform(), cfg, interp_fn=_node, apply_bc=False,
                conv_flux_fn=_flux_return_conservative)
  vec = 0.5 * np.ones(NX)
  vec[3] = 1.0
  vec[13] = 2.0
  rhs = ka.to_3d(_forward_diff(vec), 'x', SIZE)
  _check(got, {k: rhs for k in NAMES}, WIN_LO)


def flux_bc_case(kind):
  """:1484-1655 ('convective') and :1657-1826 ('total'): a uniform moving
  state (rho = 1, u = v = w = 1, T = 300 K, y = 0.5) with flux BCs on the
  x boundary faces; node face values, halo left as given, the real HLL
  flux. Returns (conserved state, cfg, expected rhs)."""
  t = 300.0
  e = orc.CV * t + 1.5
  h = orc.CP * t + 1.5
  ones = np.ones(NX)
  cons = {'rho': ones, 'rho_u': ones, 'rho_v': ones, 'rho_w': ones,
          'rho_e': e * ones, 'rho_y': 0.5 * ones}
  cons = {k: ka.to_3d(v, 'x', SIZE) for k, v in cons.items()}
  vals = {'rho': (4.0, 5.0), 'rho_v': (4.0, 5.0), 'rho_w': (4.0, 5.0),
          'rho_e': (h + 3.0, h + 4.0), 'rho_y': (3.5, 4.5)}
  spec = {}
  for k in NAMES:
    if k in vals:
      spec[k] = {'x': {0: (D, vals[k][0]), 1: (D, vals[k][1])},
                 'y': dict(NONE_SIDE), 'z': dict(NONE_SIDE)}
    else:
      spec[k] = {'x': dict(NONE_SIDE), 'y': dict(NONE_SIDE),
                 'z': dict(NONE_SIDE)}
  cfg = _cfg(dx=1.0, dy=1.0, dz=1.0)
  cfg.bc = {'intercell_fluxes': {kind: spec}}
  vec = np.ones(NX)
  vec[3] = 4.0
  vec[13] = 5.0
  rhs = ka.to_3d(_forward_diff(vec), 'x', SIZE)
  expected = {k: (np.zeros_like(rhs) if k == 'rho_u' else rhs) for k in NAMES}
  return cons, cfg, expected


@pytest.mark.parametrize('kind', ['convective', 'total'])
def test_bc_updates_intercell_fluxes_x_only(kind):
  cons, cfg, expected = flux_bc_case(kind)
  got = orc.rhs(cons, cfg, interp_fn=_node, apply_bc=False)
  _check(got, expected, WIN_LO)


def test_source_function_is_added():
  """:1828-1977: patched convective flux (returning the face values) and
  forward_1 (returning zeros); the source function returns cons + 1, so
  the rhs is cons + 1 on the interior."""
  cfg = _cfg()
  per = {d: {0: (P,), 1: (P,)} for d in ('y', 'z')}
  cfg.bc = {'cell_averages': {k: dict(per, x={0: (N, 0.0), 1: (N, 0.0)})
                              for k in NAMES}}
  vals = dict(zip(NAMES, (0.5, 1.5, 2.5, 3.5, 0.0, 4.5)))
  cons = {k: ka.to_3d(v * np.ones(NX), 'x', SIZE) for k, v in vals.items()}
  got = orc.rhs(cons, cfg, interp_fn=_node,
                conv_flux_fn=_flux_return_conservative,
                grad_fn=lambda f, h, d: np.zeros_like(f),
                source_fn=lambda c: {k: v + 1.0 for k, v in c.items()})
  _check(got, {k: ka.to_3d((v + 1.0) * np.ones(NX), 'x', SIZE)
               for k, v in vals.items()}, INTERIOR)


def test_specified_intercell_diffusive_flux():
  """:2208-2290: convective flux patched to zeros, diffusive flux patched
  to sin profiles, halo left as given."""
  flux, (xv, yv, zv) = _profiles(lambda t: np.sin(t**2.0))
  cfg = _cfg(dx=1.0, dy=1.0, dz=1.0, include_diffusion=True)
  cons = _kh_like_state(np.linspace(0.0, 1.0, NX))
  got = orc.rhs(cons, cfg, interp_fn=_node, apply_bc=False,
                conv_flux_fn=_flux_return_zeros,
                diff_flux_fn=lambda prim: flux)
  m = (ka.to_3d(_forward_diff(xv), 'x', SIZE) +
       ka.to_3d(_forward_diff(yv), 'y', SIZE) +
       ka.to_3d(_forward_diff(zv), 'z', SIZE))
  _check(got, {k: m * f for k, f in zip(NAMES, (1, 2, 3, 4, 5, 6))},
         INTERIOR)
