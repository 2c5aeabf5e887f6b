"""GPU: the unit-level CUDA kernels behind the reference's function API,
checked against the reference's known answers and against the oracle."""

import json
import os

import numpy as np
import pytest
import torch

from oracle import swirlc_oracle as orc
from tests import helpers
from tests import scenarios as sc

pytestmark = pytest.mark.gpu
DIMS = ('x', 'y', 'z')
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden',
                      'reference_vectors.json')


def _cfg(**kw):
  from swirlc_b200.core import parameter
  return parameter.SwirlCParameters(kw)


def _dev(d, dtype=torch.float64):
  return {k: torch.tensor(np.asarray(v), dtype=dtype, device='cuda')
          .reshape(1, -1, 1) for k, v in d.items()}


def _np(t):
  return t.double().cpu().numpy().reshape(-1)


@pytest.mark.parametrize('dim', DIMS)
def test_wave_speeds_known_answers(dim):
  from swirlc_b200.numerics.riemann_solver import hll, hllc
  cfg = _cfg()
  c = sc.uniform(dim)
  s_l, s_r = hll.compute_hll_roe_wave_speed_estimates(
      0, np.array([[[0]]]), _dev(c['neg']), _dev(c['pos']), dim, cfg, None)
  np.testing.assert_allclose(_np(s_l), c['s_l'], rtol=1e-12)
  np.testing.assert_allclose(_np(s_r), c['s_r'], rtol=1e-12)
  _, s_m, _ = hllc._compute_wave_speeds(0, np.array([[[0]]]), _dev(c['neg']),
                                        _dev(c['pos']), dim, cfg, None)
  np.testing.assert_allclose(_np(s_m), c['s_m'], rtol=1e-12)
  for left in (True, False):
    c = sc.shock_speeds(dim, left)
    for dtype, tol in ((torch.float64, 1e-9), (torch.float32, 2e-6)):
      s_l, s_r = hll.compute_hll_roe_wave_speed_estimates(
          0, np.array([[[0]]]), _dev(c['neg'], dtype), _dev(c['pos'], dtype),
          dim, cfg, None)
      np.testing.assert_allclose(_np(s_l), c['s_l'], rtol=tol)
      np.testing.assert_allclose(_np(s_r), c['s_r'], rtol=tol)


@pytest.mark.parametrize('case', sorted(sc.FLUX_CASES))
@pytest.mark.parametrize('solver', ['hll', 'hllc'])
@pytest.mark.parametrize('dim', DIMS)
@pytest.mark.parametrize('dtype', [torch.float64, torch.float32])
def test_riemann_flux_known_answers(dtype, dim, solver, case):
  from swirlc_b200.numerics.riemann_solver import riemann_solver
  cfg = _cfg(numeric_flux_scheme=solver.upper())
  fn = riemann_solver.select_numeric_flux_fn(cfg)
  c = sc.FLUX_CASES[case](dim)
  got = fn(0, np.array([[[0]]]), _dev(c['cneg'], dtype), _dev(c['cpos'], dtype),
           _dev(c['neg'], dtype), _dev(c['pos'], dtype), {}, {}, None, dim, cfg,
           None)
  # float32 uses the fast-math division/sqrt (<= 2 ulp each); float64 keeps
  # FMA contraction (a few ulp on differences of products).
  rtol = 1e-9 if dtype == torch.float64 else 2e-5
  # Errors are measured against the case's flux scale (symmetric cases cancel
  # to rounding level of that scale).
  scale = max(max(np.abs(w).max() for w in c['flux'].values()), 1.0)
  for k, want in c['flux'].items():
    np.testing.assert_allclose(_np(got[k]), want, rtol=rtol,
                               atol=rtol * scale, err_msg=f'{solver} {case} {k}')


@pytest.mark.parametrize('solver', ['HLL', 'HLLC'])
def test_riemann_flux_with_scalar_matches_oracle(solver):
  from swirlc_b200.numerics.riemann_solver import riemann_solver
  cfg = _cfg(numeric_flux_scheme=solver,
             conservative_variable_names=list(orc.BASE_CONSERVATIVE) + ['rho_y'])
  rng = np.random.default_rng(3)
  n = 512

  def side(seed):
    r = np.random.default_rng(seed)
    rho = r.uniform(0.2, 2.0, n)
    u, v, w = (r.uniform(-2, 2, n) for _ in range(3))
    p = r.uniform(0.2, 5.0, n)
    y = r.uniform(0, 1, n)
    prim, cons = sc.state(rho, (u, v, w), p, p / (orc.R * rho))
    prim['y'] = y
    cons['rho_y'] = rho * y
    return prim, cons

  pn, cn = side(1)
  pp, cp = side(2)
  del rng
  for dim in DIMS:
    got = riemann_solver.select_numeric_flux_fn(cfg)(
        0, np.array([[[0]]]), _dev(cn), _dev(cp), _dev(pn), _dev(pp), {}, {},
        None, dim, cfg, None)
    fn = orc.hll_flux if solver == 'HLL' else orc.hllc_flux
    want = fn(cn, cp, pn, pp, {}, {}, dim, list(cfg.conservative_variable_names),
              0.0)
    for k in want:
      np.testing.assert_allclose(_np(got[k]), want[k], rtol=1e-9, atol=1e-9,
                                 err_msg=f'{dim} {k}')


def test_gradient_golden_vectors():
  from swirlc_b200.numerics import gradient
  with open(GOLDEN) as f:
    gold = json.load(f)
  x = np.linspace(0, 2.0 * np.pi, 16)
  h = x[1] - x[0]
  for dim in DIMS:
    f3 = torch.tensor(helpers.to_3d(np.sin(x), dim, (16, 16, 16)),
                      dtype=torch.float32, device='cuda')
    sel = {'x': (8, slice(None), 8), 'y': (8, 8, slice(None)),
           'z': (slice(None), 8, 8)}[dim]
    fwd = gradient.forward_1(f3, h, dim).cpu().numpy()[sel]
    np.testing.assert_allclose(fwd[:-1], gold['gradient_forward_1'],
                               rtol=1e-5, atol=1e-5)
    cen = gradient.central_2(f3, h, dim).cpu().numpy()[sel]
    np.testing.assert_allclose(cen[1:-1], gold['gradient_central_2'],
                               rtol=1e-5, atol=1e-5)
    bwd = gradient.backward_1(f3, h, dim).cpu().numpy()[sel]
    exp = np.zeros(16)
    exp[1:] = np.diff(np.sin(x)) / h
    np.testing.assert_allclose(bwd[1:], exp[1:], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize('dim', DIMS)
def test_linear_interpolation(dim):
  from swirlc_b200.numerics import interpolation
  f = np.logspace(0.0, 2.0, 16)
  f3 = torch.tensor(helpers.to_3d(f, dim, (16, 16, 16)), device='cuda')
  for fd in DIMS:
    got = interpolation.linear_interpolation(f3, fd).cpu().numpy()
    want = orc.linear_interpolation(helpers.to_3d(f, dim, (16, 16, 16)), fd)
    np.testing.assert_allclose(got[1:, 1:, 1:], want[1:, 1:, 1:], rtol=1e-14)


@pytest.mark.parametrize('scheme', ['weno5', 'weno3', 'mc', 'van_leer',
                                    'minmod', 'minmod3'])
@pytest.mark.parametrize('dtype', [torch.float32, torch.float64])
def test_reconstruction_matches_oracle(scheme, dtype):
  from swirlc_b200.numerics import interpolation
  rng = np.random.default_rng(7)
  npd = np.float32 if dtype == torch.float32 else np.float64
  v = (np.sin(np.linspace(0, 6, 20))[None, :, None] * np.ones((14, 20, 18))
       + 0.3 * rng.random((14, 20, 18))).astype(npd)
  vt = torch.tensor(v, device='cuda')
  for dim in DIMS:
    if scheme == 'weno5':
      got, want = interpolation.weno(vt, dim, 3), orc.weno(v, dim, 3)
    elif scheme == 'weno3':
      got, want = interpolation.weno(vt, dim, 2), orc.weno(v, dim, 2)
    else:
      lt = {'mc': interpolation.FluxLimiterType.MUSCL,
            'van_leer': interpolation.FluxLimiterType.VAN_LEER,
            'minmod': interpolation.FluxLimiterType.MINMOD,
            'minmod3': interpolation.FluxLimiterType.MINMOD3}[scheme]
      got, want = interpolation.flux_limiter(vt, dim, lt), orc.muscl(v, dim,
                                                                     scheme)
    tol = 2e-6 if dtype == torch.float32 else 1e-12
    ax = orc.AXIS[dim]
    sl = [slice(None)] * 3
    sl[ax] = slice(3, -3)
    sl = tuple(sl)
    for g, w in zip(got, want):
      np.testing.assert_allclose(g.cpu().numpy()[sl], w[sl], rtol=tol,
                                 atol=tol, err_msg=f'{scheme} {dim}')


@pytest.mark.parametrize('dtype', [torch.float32, torch.float64])
def test_van_leer_extreme_ratios_stay_finite(dtype):
  """Float64 keeps subnormals: beside a subnormal value dm / dp is +-inf or
  a finite ratio whose r + |r| overflows (lines seen in the buoyant bubble
  run in float64). From |r| >= 2^54 (2^25 in float32) van Leer's phi is
  exactly 2 or 0, on the GPU and in the oracle alike, never inf or NaN."""
  from swirlc_b200.numerics import interpolation
  if dtype == torch.float64:
    line = [5.67e-16, -1.41e-16, 7.9e-16, 5e-324, 0.0, 0.0, -5.70e-15,
            5e-324, 0.0, -5e-324, 3e-15, 0.0, 5e-324, -5e-324, 1e-16, 2e-16]
  else:
    line = [0.5, -0.2, 5.0, 1.2e-38, 0.0, 0.0, -1.2e-38, 3.0, 0.0, 1.5e-38,
            0.1, -4.0, -1.2e-38, 0.0, 0.2, 0.3]
  npd = np.float64 if dtype == torch.float64 else np.float32
  line = np.array(line, npd)
  v = np.broadcast_to(line[None, None, :], (10, 10, line.size)).copy()
  vt = torch.tensor(v, device='cuda')
  got = interpolation.flux_limiter(vt, 'y',
                                   interpolation.FluxLimiterType.VAN_LEER)
  with np.errstate(over='ignore', divide='ignore'):
    want = orc.muscl(v, 'y', 'van_leer')
  # float32 runs flush-to-zero: values below its smallest normal may differ.
  tol, atol = (1e-12, 1e-300) if dtype == torch.float64 else (2e-6, 1e-37)
  sl = (slice(None), slice(None), slice(3, -3))
  for g, w in zip(got, want):
    g = g.cpu().numpy()[sl]
    assert np.isfinite(g).all() and np.isfinite(w[sl]).all()
    np.testing.assert_allclose(g, w[sl], rtol=tol, atol=atol)


def test_exchange_halos_matches_boundary_test():
  """boundary_test.py:60-343 (single replica) through the CUDA halo fill."""
  from swirlc_b200.boundary import bc_types, boundary
  BC = bc_types.BoundaryCondition
  n = 16
  u0 = np.zeros((n, n, n), np.float32)
  u0[3:-3, 3:-3, 3:-3] = 6.0
  p0 = np.zeros((n, n, n), np.float32)
  p0[3:-3, 3:-3, 3:-3] = 200.0
  u_bc_z0 = [np.ones((n, n)), 2.0 * np.ones((n, n)), 3.0 * np.ones((n, n))]
  p_bc_x1 = [[60.0 * np.ones((1, n))] * n, [80.0 * np.ones((1, n))] * n,
             [120.0 * np.ones((1, n))] * n]
  cfg = _cfg(halo_width=3, bc={
      'u': {'x': {0: (BC.DIRICHLET, 8.0), 1: (BC.NEUMANN, 0.0)},
            'y': {0: (BC.PERIODIC,), 1: (BC.PERIODIC,)},
            'z': {0: (BC.DIRICHLET, u_bc_z0), 1: (BC.NEUMANN, 1.0)}},
      'p': {'x': {0: (BC.NEUMANN, 8.0), 1: (BC.DIRICHLET, p_bc_x1)},
            'y': {0: (BC.PERIODIC,), 1: (BC.PERIODIC,)},
            'z': {0: (BC.DIRICHLET, 100.0), 1: (BC.NEUMANN, 0.0)}}})
  out = boundary.update_boundary(
      0, np.array([[[0]]]),
      {'u': list(torch.unbind(torch.tensor(u0, device='cuda'))),
       'p': torch.tensor(p0, device='cuda')}, cfg)
  u = torch.stack(out['u']).cpu().numpy()
  p = out['p'].cpu().numpy()
  i = slice(3, -3)
  np.testing.assert_array_equal(u[i, :3, i], 8.0)
  np.testing.assert_array_equal(u[i, -3:, i], 6.0)
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
  # Whole arrays, corners and edges included, against the oracle.
  bc_u = {'x': {0: (orc.DIRICHLET, 8.0), 1: (orc.NEUMANN, 0.0)},
          'y': {0: (orc.PERIODIC,), 1: (orc.PERIODIC,)},
          'z': {0: (orc.DIRICHLET, u_bc_z0), 1: (orc.NEUMANN, 1.0)}}
  bc_p = {'x': {0: (orc.NEUMANN, 8.0),
                1: (orc.DIRICHLET, [np.full((n, n), v) for v in
                                    (60.0, 80.0, 120.0)])},
          'y': {0: (orc.PERIODIC,), 1: (orc.PERIODIC,)},
          'z': {0: (orc.DIRICHLET, 100.0), 1: (orc.NEUMANN, 0.0)}}
  np.testing.assert_array_equal(u, orc.exchange_halos(u0, bc_u, 3))
  np.testing.assert_array_equal(p, orc.exchange_halos(p0, bc_p, 3))


def test_conservative_cell_averages_primitive_bc():
  """boundary_test.py:345-561 (one replica): a velocity BC given on the
  primitive is applied to rho_u/rho and multiplied by the updated rho."""
  from swirlc_b200.boundary import bc_types, boundary
  BC = bc_types.BoundaryCondition
  n = 16
  per = {0: (BC.PERIODIC,), 1: (BC.PERIODIC,)}
  rho_f0 = [1.0, 2.0, 3.0]
  u_f0 = [11.0, 21.0, 31.0]
  bc = {
      'rho': {'x': {0: (BC.DIRICHLET, rho_f0), 1: (BC.NEUMANN, 0.0)},
              'y': per, 'z': per},
      'u': {'x': {0: (BC.DIRICHLET, u_f0), 1: (BC.NEUMANN, 0.0)},
            'y': per, 'z': per},
      'rho_v': {'x': {0: (BC.DIRICHLET, [-12.0, -22.0, -32.0]),
                      1: (BC.NEUMANN, 0.0)}, 'y': per, 'z': per},
      'rho_w': {'x': {0: (BC.DIRICHLET, [13.0, 23.0, 33.0]),
                      1: (BC.NEUMANN, 0.0)}, 'y': per, 'z': per},
      'rho_e': {'x': {0: (BC.DIRICHLET, [15.0, 25.0, 35.0]),
                      1: (BC.NEUMANN, 1.0)}, 'y': per, 'z': per},
  }
  cfg = _cfg(halo_width=3, bc={'cell_averages': bc})
  vals = {'rho': 1.0, 'rho_u': 2.0, 'rho_v': 3.0, 'rho_w': 4.0, 'rho_e': 5.0}
  cons = {k: torch.full((n, n, n), v, dtype=torch.float64, device='cuda')
          for k, v in vals.items()}
  out = boundary.update_conservative_cell_averages(0, np.array([[[0]]]), cons,
                                                   cfg)
  o = {k: v.cpu().numpy() for k, v in out.items()}
  for l in range(3):
    np.testing.assert_allclose(o['rho'][:, l, :], rho_f0[l])
    np.testing.assert_allclose(o['rho_u'][:, l, :], rho_f0[l] * u_f0[l])
  np.testing.assert_allclose(o['rho_u'][:, -3:, :], 2.0)
  np.testing.assert_allclose(o['rho_e'][:, -3:, :][:, 0, :], 6.0)
  np.testing.assert_allclose(o['rho_e'][:, -1, :], 8.0)


def test_rk3_user_rhs_stage_algebra():
  """rk3_test.py:92-213 through the stage-combination kernel."""
  from swirlc_b200.numerics.time_integration import rk3, rk2
  cfg = _cfg(dt=0.1, halo_width=0)
  names = list(orc.BASE_CONSERVATIVE) + ['rho_y']
  s0 = {k: torch.full((4, 4, 4), float(i + 1), dtype=torch.float64,
                      device='cuda') for i, k in enumerate(names)}

  def rhs_const(rid, st, hv):
    return {k: torch.zeros_like(v) for k, v in st.items()}

  def rhs_stage(rid, st, hv):
    m = float(st['rho'].mean())
    f = 20.0 if m < 2.0 else (40.0 if m > 2.75 else -10.0)
    return {k: torch.full_like(v, f) for k, v in st.items()}

  out = rk3.integrate(0, None, s0, {}, cfg, None, rhs_const)
  for k in names:
    np.testing.assert_allclose(out[k].cpu().numpy(), s0[k].cpu().numpy(),
                               rtol=4e-16)
  out = rk3.integrate(0, None, s0, {}, cfg, None, rhs_stage)
  for k in names:
    np.testing.assert_allclose(out[k].cpu().numpy(),
                               s0[k].cpu().numpy() + 1.0 / 3.0, rtol=1e-12)
  # rk2_test.py:85-207: the same state and constant rhs give u0 + dt*f.
  out = rk2.integrate(0, None, s0, {}, cfg, None,
                      lambda r, s, h: {k: torch.full_like(v, 5.0)
                                       for k, v in s.items()})
  for k in names:
    np.testing.assert_allclose(out[k].cpu().numpy(),
                               s0[k].cpu().numpy() + 0.5, rtol=1e-12)


def test_time_integration_rejects_unknown_scheme():
  from swirlc_b200.numerics.time_integration import time_integration
  cfg = _cfg(time_integration_scheme='rk4')
  with pytest.raises(NotImplementedError):
    time_integration.time_integration(0, None, {}, {}, cfg, None, None)


@pytest.mark.parametrize('dim,v_conv', [('x', 10.0), ('y', -25.0),
                                        ('z', 15.0)])
def test_fused_rhs_plug_flow_with_identity_faces(dim, v_conv):
  """compressible_navier_stokes_test.py:976-1053 through the fused kernel
  (identity face values as the reference's WENO mock, periodic halos)."""
  from swirlc_b200.equations import compressible_navier_stokes as cns
  from swirlc_b200.physics import physics_models
  n = 16
  p = 101325.0 * np.ones(n)
  t = 300.0 * np.ones(n)
  rho = p / (orc.R * t)
  vel = [np.zeros(n)] * 3
  vel = list(vel)
  vel[DIMS.index(dim)] = v_conv * np.ones(n)
  e = orc.CV * t + 0.5 * (vel[0]**2 + vel[1]**2 + vel[2]**2)
  cons = {'rho': rho, 'rho_u': rho * vel[0], 'rho_v': rho * vel[1],
          'rho_w': rho * vel[2], 'rho_e': rho * e}
  cfg = _cfg(interpolation_scheme='NODE', numeric_flux_scheme='HLL')
  rhs = cns.get_rhs_fn(np.array([[[0]]]), cfg,
                       physics_models.PhysicsModels(cfg))
  dev = {k: torch.tensor(helpers.to_3d(v, dim, (n, n, n)), device='cuda')
         for k, v in cons.items()}
  out = rhs(0, dev, {})
  for k, v in out.items():
    scale = max(np.abs(cons[k]).max(), 1.0) / cfg.dx
    np.testing.assert_allclose(v.cpu().numpy()[3:-3, 3:-3, 3:-3], 0.0,
                               atol=1e-9 * scale, err_msg=k)


@pytest.mark.parametrize('scheme', ['WENO_5', 'WENO_3', 'MUSCL', 'NODE'])
@pytest.mark.parametrize('flux', ['HLL', 'HLLC'])
def test_fused_rhs_quiescent_gas_is_zero(scheme, flux):
  """compressible_navier_stokes_test.py:927-966 for every scheme."""
  from swirlc_b200.equations import compressible_navier_stokes as cns
  from swirlc_b200.physics import physics_models
  cfg = _cfg(interpolation_scheme=scheme, numeric_flux_scheme=flux)
  rhs = cns.get_rhs_fn(np.array([[[0]]]), cfg,
                       physics_models.PhysicsModels(cfg))
  p, t = 101325.0, 500.0
  rho = p / (orc.R * t)
  cons = {'rho': rho, 'rho_u': 0.0, 'rho_v': 0.0, 'rho_w': 0.0,
          'rho_e': rho * orc.CV * t}
  dev = {k: torch.full((16, 16, 16), v, dtype=torch.float64, device='cuda')
         for k, v in cons.items()}
  out = rhs(0, dev, {})
  for k, v in out.items():
    assert float(v[3:-3, 3:-3, 3:-3].abs().max()) < 1e-6, k


def test_select_numeric_flux_fn_errors():
  from swirlc_b200.numerics.riemann_solver import riemann_solver, hll
  assert riemann_solver.select_numeric_flux_fn(_cfg()) is hll.hll_convective_flux
  with pytest.raises(ValueError):
    riemann_solver.select_numeric_flux_fn(_cfg(numeric_flux_scheme='ROE'))


@pytest.mark.parametrize('modes,shape', [
    (('neumann0', 'periodic', 'periodic'), (14, 22, 12)),
    (('periodic', 'periodic', 'periodic'), (12, 9, 10)),
    (('neumann0', 'neumann0', 'neumann0'), (10, 12, 14)),
    (('periodic', 'neumann0', 'neumann0'), (9, 9, 9)),  # interior 3 = halo
])
def test_one_pass_halo_fill_matches_three_passes(modes, shape):
  """Grids whose every dim is periodic or zero-gradient take the one-pass
  halo fill (each halo cell copies the interior cell it wraps or clamps
  to); the result must equal the oracle's x, y, z passes bit for bit,
  corners and edges included, whatever the halos held before."""
  from swirlc_b200.boundary import bc_types, boundary
  BC = bc_types.BoundaryCondition
  rng = np.random.default_rng(7)
  spec = {'periodic': ((BC.PERIODIC,), (BC.PERIODIC,)),
          'neumann0': ((BC.NEUMANN, 0.0), (BC.NEUMANN, 0.0))}
  ospec = {'periodic': ((orc.PERIODIC,), (orc.PERIODIC,)),
           'neumann0': ((orc.NEUMANN, 0.0), (orc.NEUMANN, 0.0))}
  dims = ('x', 'y', 'z')
  bc = {d: {0: spec[m][0], 1: spec[m][1]} for d, m in zip(dims, modes)}
  obc = {d: {0: ospec[m][0], 1: ospec[m][1]} for d, m in zip(dims, modes)}
  names = ('u', 'v', 'p')
  cfg = _cfg(halo_width=3, bc={k: bc for k in names})
  init = {k: rng.standard_normal(shape).astype(np.float32) for k in names}
  out = boundary.update_boundary(
      0, np.array([[[0]]]),
      {k: torch.tensor(v, device='cuda') for k, v in init.items()}, cfg)
  for k in names:
    np.testing.assert_array_equal(out[k].cpu().numpy(),
                                  orc.exchange_halos(init[k], obc, 3))


@pytest.mark.parametrize('dtype', [np.float32, np.float64])
@pytest.mark.parametrize('shape', [(14, 22, 12), (9, 11, 10)])
def test_composed_one_pass_halo_fill_matches_three_passes(dtype, shape):
  """Fields whose sides mix periodic, Dirichlet (values and per-layer
  planes) and Neumann (nonzero increments) take the composed one-pass fill
  (each halo cell walks the passes back to its source); the result must
  equal the oracle's x, y, z passes bit for bit, corners and edges
  included, whatever the halos held before."""
  from swirlc_b200.boundary import bc_types, boundary
  BC = bc_types.BoundaryCondition
  rng = np.random.default_rng(11)
  hw = 3
  dims = ('x', 'y', 'z')
  plane_shape = {'x': (shape[0], shape[2]), 'y': (shape[0], shape[1]),
                 'z': (shape[1], shape[2])}

  def side(d, kind):
    if kind == 'dirichlet':
      v = float(rng.uniform(-2.0, 2.0))
      return (BC.DIRICHLET, v), (orc.DIRICHLET, v)
    if kind == 'planes':
      pl = [rng.standard_normal(plane_shape[d]).astype(dtype)
            for _ in range(hw)]
      return (BC.DIRICHLET, pl), (orc.DIRICHLET, pl)
    v = float(rng.uniform(-1.0, 1.0))
    return (BC.NEUMANN, v), (orc.NEUMANN, v)

  kinds = ('dirichlet', 'planes', 'neumann')
  names = ('u', 'v', 'p', 'q')
  bc, obc = {}, {}
  for i, k in enumerate(names):
    bc[k], obc[k] = {}, {}
    for j, d in enumerate(dims):
      if (i + j) % 3 == 0:
        bc[k][d] = {0: (BC.PERIODIC,), 1: (BC.PERIODIC,)}
        obc[k][d] = {0: (orc.PERIODIC,), 1: (orc.PERIODIC,)}
        continue
      lo, olo = side(d, kinds[(i + 2 * j) % 3])
      hi, ohi = side(d, kinds[(i + j + 1) % 3])
      bc[k][d] = {0: lo, 1: hi}
      obc[k][d] = {0: olo, 1: ohi}
  cfg = _cfg(halo_width=hw, bc=bc)
  init = {k: rng.standard_normal(shape).astype(dtype) for k in names}
  out = boundary.update_boundary(
      0, np.array([[[0]]]),
      {k: torch.tensor(v, device='cuda') for k, v in init.items()}, cfg)
  for k in names:
    np.testing.assert_array_equal(out[k].cpu().numpy(),
                                  orc.exchange_halos(init[k], obc[k], hw),
                                  err_msg=k)
