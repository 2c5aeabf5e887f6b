"""GPU: a grid decomposed into blocks (replicas cx x cy x cz), stepped block
by block with halo exchange between the blocks in this process, ends bit for
bit where the single-grid run ends (same dt from the min-reduced CFL
limit)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NAMES = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')


def _single(cfg, state, steps, dtype, scheme):
  from swirlc_b200 import engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  p = parameter.SwirlCParameters(cfg)
  s = engine.Solver(p, physics_models.PhysicsModels(p), state['rho'].shape,
                    dtype)
  f = [torch.as_tensor(state[k]).to('cuda', dtype).contiguous() for k in NAMES]
  st = engine.Stepper(s, f, dt=p.dt, cfl=p.cfl, t_end=p.t_end, scheme=scheme)
  st.step(steps)
  torch.cuda.synchronize()
  hw = p.halo_width
  return ({k: v[hw:-hw, hw:-hw, hw:-hw].cpu().numpy()
           for k, v in zip(NAMES, f)}, st.clock.cpu())


def _decomposed(cfg, state, shape, steps, dtype, scheme, overlap=None):
  from swirlc_b200 import decomposition
  cfg = dict(cfg, cx=shape[0], cy=shape[1], cz=shape[2])
  replicas = np.arange(int(np.prod(shape))).reshape(shape)
  hw = cfg['halo_width']
  blocks = decomposition.split_state(state, replicas, hw)
  ds = decomposition.DecomposedStepper(cfg, blocks, dtype=dtype,
                                       transport='local', scheme=scheme,
                                       overlap=bool(overlap))
  if overlap is not None:
    assert ds.overlap == overlap
  ds.step(steps)
  out = decomposition.join_interiors(ds.states(), replicas, hw)
  return out, [c.cpu() for c in ds.clocks]


def _check(cfg, state, shape, steps=3, dtype=torch.float32, scheme='rk3',
           overlap=None):
  want, clock = _single(cfg, state, steps, dtype, scheme)
  got, clocks = _decomposed(cfg, state, shape, steps, dtype, scheme, overlap)
  for k in NAMES:
    assert np.array_equal(got[k], want[k]), (shape, k,
                                             np.abs(got[k] - want[k]).max())
  for c in clocks:
    assert torch.equal(c, clock)


@pytest.mark.parametrize('shape', [(2, 2, 1), (1, 2, 2), (2, 1, 3)])
def test_kh_viscous_blocks_match_single_grid(shape):
  from swirlc_b200 import configs
  cfg, state = configs.kelvin_helmholtz(n=24, nu=1e-3)
  _check(cfg, state, shape)


def test_sod_neumann_walls_four_blocks():
  from swirlc_b200 import configs
  cfg, state = configs.sod(n=64, ny=8, nz=8)
  _check(cfg, state, (4, 1, 1), steps=5)


def test_bubble_gravity_dirichlet_planes_split_along_gravity_rk2_f64():
  from swirlc_b200 import configs
  cfg, state = configs.buoyant_bubble(nx=12, ny=10, nz=16)
  _check(cfg, state, (1, 1, 2), steps=3, dtype=torch.float64, scheme='rk2')


def test_bubble_muscl_hll_split_across_gravity_f32():
  from swirlc_b200 import configs
  cfg, state = configs.buoyant_bubble(nx=16, ny=8, nz=12)
  _check(cfg, state, (2, 2, 1), steps=3)


@pytest.mark.parametrize('shape', [(2, 1, 1), (1, 2, 2)])
def test_overlapped_halo_update_matches_single_grid(shape):
  """Halo update on a side stream behind the inner boxes' stage, then the
  shell boxes: bit for bit the single-grid run."""
  from swirlc_b200 import configs
  cfg, state = configs.kelvin_helmholtz(n=80, nu=1e-3)
  _check(cfg, state, shape, steps=2, overlap=True)


def test_overlapped_halo_update_with_walls_and_gravity():
  from swirlc_b200 import configs
  cfg, state = configs.buoyant_bubble(nx=80, ny=36, nz=80, lz=100.0)
  _check(cfg, state, (2, 1, 2), steps=2, overlap=True)


@pytest.mark.parametrize('dtype', [torch.float32, torch.float64])
def test_sub_box_stages_partition_the_whole_stage(dtype):
  """stage_box on the inner box and the six shell boxes of split_boxes
  gives the whole stage (and its CFL limit) bit for bit."""
  from swirlc_b200 import _native as nat
  from swirlc_b200 import configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  cfg, state = configs.kelvin_helmholtz(n=40, nu=1e-3)
  p = parameter.SwirlCParameters(cfg)
  s = engine.Solver(p, physics_models.PhysicsModels(p), state['rho'].shape,
                    dtype)
  u = [torch.tensor(state[k], dtype=dtype, device='cuda') for k in NAMES]
  s.fill_halos(u)
  dt = s.dt_tensor(1e-3)
  inner, shell = s.split_boxes()
  assert inner == (16, 24, 16, 24, 3, 37) and len(shell) == 6
  whole, parts = s.new_fields(), s.new_fields()
  m1 = torch.full((1,), 1e300, dtype=torch.float64, device='cuda')
  m2 = m1.clone()
  s.stage(u, u, whole, nat.SWC_OUT_CONVEX, 0.75, 0.25, dt=dt, dtmin_out=m1)
  for box in [inner] + shell:
    s.stage_box(u, u, parts, nat.SWC_OUT_CONVEX, box, 0.75, 0.25, dt=dt,
                dtmin_out=m2)
  sl = (slice(3, -3),) * 3
  for a, b in zip(whole, parts):
    assert torch.equal(a[sl], b[sl])
  assert torch.equal(m1, m2)
  with pytest.raises(ValueError):
    s.stage_box(u, u, parts, nat.SWC_OUT_CONVEX, (0, 41, 0, 8, 0, 8))


@pytest.mark.parametrize('zseg', [1, 3, 5])
def test_stage_results_do_not_depend_on_z_segments(zseg):
  """Each CTA marches over zseg planes; the face below its first plane is
  computed by the same code as every other face, so any zseg gives the same
  bits."""
  from swirlc_b200 import configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  cfg, state = configs.kelvin_helmholtz(n=20, nu=1e-3)
  p = parameter.SwirlCParameters(cfg)
  outs = []
  for zs in (0, zseg):
    s = engine.Solver(p, physics_models.PhysicsModels(p), state['rho'].shape)
    s.scheme.zseg = zs
    f = [torch.tensor(state[k], device='cuda') for k in NAMES]
    outs.append(s.rk3(f, 1e-3))
  for a, b in zip(*outs):
    assert torch.equal(a[3:-3, 3:-3, 3:-3], b[3:-3, 3:-3, 3:-3])


def test_decomposed_stepper_argument_errors():
  from swirlc_b200 import configs, decomposition
  cfg, state = configs.kelvin_helmholtz(n=16)
  cfg = dict(cfg, cx=2)
  blocks = decomposition.split_state(state, np.arange(2).reshape(2, 1, 1), 3)
  with pytest.raises(ValueError):
    decomposition.DecomposedStepper(cfg, {0: blocks[0]}, transport='local')
  with pytest.raises(ValueError):
    decomposition.DecomposedStepper(cfg, blocks, transport='dist')
