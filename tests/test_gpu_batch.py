"""GPU: batched time step (swc_batch_step) of many independent grids.

Each member of a batch must end bit for bit where the single-grid step
(swc_rk_step through engine.Stepper) takes it, with its own CFL time step;
small members are also checked against the oracle."""

import numpy as np
import pytest
import torch

from helpers import rel_l2

pytestmark = pytest.mark.gpu

NAMES = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')


def _single(cfg, state, steps, dtype=torch.float32, scheme='rk3', cfl=None):
  from swirlc_b200 import engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  p = parameter.SwirlCParameters(cfg)
  solver = engine.Solver(p, physics_models.PhysicsModels(p),
                         state['rho'].shape, dtype)
  f = [torch.as_tensor(state[k]).to('cuda', dtype).contiguous() for k in NAMES]
  c = float(p.cfl if cfl is None else cfl)
  st = engine.Stepper(solver, f, dt=float(p.dt), cfl=c, scheme=scheme)
  st.step(steps)
  return f, st.clock


def _compare(batch, members, steps, dtype=torch.float32, scheme='rk3',
             exact=None):
  """Bit for bit where member i ran 16x16 tiles (exact[i] true, the default),
  else within 1e-6 relative L2 (the 8x32 tile rounds differently)."""
  for i, (cfg, state) in enumerate(members):
    ref, clock = _single(cfg, state, steps, dtype, scheme)
    hw = batch.solvers[i].hw
    sl = (slice(hw, -hw),) * 3
    bitwise = exact is None or exact[i]
    for name, a, b in zip(NAMES, batch.u[i], ref):
      if bitwise:
        assert torch.equal(a[sl], b[sl]), (i, name)
      else:
        err = rel_l2(a.double().cpu().numpy(), b.double().cpu().numpy(), hw)
        assert err <= 1e-6, (i, name, err)
    if bitwise:
      assert torch.equal(batch.clocks[i], clock), i
    else:
      assert batch.clocks[i].tolist()[:3] == pytest.approx(
          clock.tolist()[:3], rel=1e-5), i


def test_riemann_batch_matches_single_grid_steps():
  """The 64 seeded quasi-1-D Riemann problems, 3 steps, own CFL dt each."""
  from swirlc_b200 import batch, configs
  members = configs.riemann_batch()
  b = batch.BatchStepper(members)
  b.step(3)
  torch.cuda.synchronize()
  _compare(b, members, 3)
  dts = sorted({float(c[1]) for c in b.clocks})
  assert len(dts) > 32  # every member took its own time step


def test_batch_graph_replay_and_forced_launch_shapes():
  from swirlc_b200 import batch, configs
  members = configs.riemann_batch(members=12, seed=5)
  b = batch.BatchStepper(members)
  # 16x16 for the narrow members, 8x32 for the wide ones, odd z segments.
  tiles = [batch.TILE_16X16 if s.ny <= 8 else batch.TILE_8X32
           for s in b.solvers]
  b.set_launch(tiles, [3] * b.n_members)
  b.step(1)
  b.capture(steps=2)
  b.step(4)
  torch.cuda.synchronize()
  _compare(b, members, 5, exact=[t == batch.TILE_16X16 for t in tiles])


def test_batch_autotune_keeps_state():
  from swirlc_b200 import batch, configs
  members = configs.riemann_batch(members=10, seed=7)
  b = batch.BatchStepper(members)
  before = [[f.clone() for f in u] for u in b.u]
  res = b.autotune(steps=1, reps=1)
  assert len(res['results']) == 8 and res['ms_per_step'] > 0
  for u, v in zip(b.u, before):
    assert all(torch.equal(x, y) for x, y in zip(u, v))
  assert all(int(c[5:6].view(torch.int64)) == 0 for c in b.clocks)
  b.step(2)
  torch.cuda.synchronize()
  exact = [b.table[i].tile != batch.TILE_8X32 for i in range(b.n_members)]
  _compare(b, members, 2, exact=exact)


def test_batch_viscous_gravity_rk2_float64():
  """Members with viscous fluxes, gravity (potential energy along z),
  Dirichlet per-layer planes and RK2, in double."""
  from swirlc_b200 import batch, configs
  members = []
  for nx, ny, nz in ((20, 16, 12), (36, 8, 10), (12, 24, 20)):
    cfg, state = configs.buoyant_bubble(nx=nx, ny=ny, nz=nz)
    cfg = dict(cfg, include_diffusion=True, dt=2e-4,
               transport_parameters={'nu': 1e-3, 'pr': 0.7})
    members.append((cfg, state))
  b = batch.BatchStepper(members, dtype=torch.float64, scheme='rk2')
  b.step(2)
  torch.cuda.synchronize()
  _compare(b, members, 2, torch.float64, 'rk2')


def test_batch_one_step_matches_oracle():
  from oracle import swirlc_oracle as orc
  from swirlc_b200 import batch, configs
  keys = ('halo_width', 'dx', 'dy', 'dz', 'interpolation_scheme',
          'numeric_flux_scheme', 'include_diffusion', 'transport_parameters',
          'muscl_limiter', 'x', 'y', 'z', 'bc', 'g', 'source_functions')
  members = [m for m in configs.riemann_batch(members=24, seed=1)
             if m[1]['rho'].size <= 60000][:4]
  assert len(members) >= 2
  b = batch.BatchStepper(members)
  b.step(1)
  torch.cuda.synchronize()
  for i, (cfg, state) in enumerate(members):
    dt = np.float32(float(b.clocks[i][1]))
    ocfg = orc.make_cfg(**{k: cfg[k] for k in keys if k in cfg})
    s0 = {k: np.asarray(state[k], np.float32) for k in NAMES}
    ref = orc.rk3(s0, dt, lambda u: orc.rhs(u, ocfg))
    hw = cfg['halo_width']
    for name, a in zip(NAMES, b.u[i]):
      got = a.double().cpu().numpy()
      want = np.asarray(ref[name], np.float64)
      if np.linalg.norm(want[hw:-hw, hw:-hw, hw:-hw]) == 0.0:
        assert np.abs(got[hw:-hw, hw:-hw, hw:-hw]).max() <= 1e-6, (i, name)
      else:
        err = rel_l2(got, want, hw)
        assert err <= 1e-5, (i, name, err)


def test_batch_rejects_bad_members():
  import ctypes
  from swirlc_b200 import _native as nat
  from swirlc_b200 import batch, configs
  members = configs.riemann_batch(members=2, seed=2)
  b = batch.BatchStepper(members)
  b.table[1].tile = 7
  with pytest.raises(ValueError, match='tile'):
    b.step(1)
  b.table[1].tile = 0
  b.table[0].grid.halo = 2
  with pytest.raises(ValueError, match='halo'):
    b.step(1)
  b.table[0].grid.halo = 3
  with pytest.raises(NotImplementedError):
    nat.check(nat.load().swc_batch_step(ctypes.byref(b.scheme), 4, 2, b.table,
                                        nat.stream_ptr()))
  other = configs.riemann_batch(members=1, seed=3)[0]
  cfg = dict(other[0], numeric_flux_scheme='HLL')
  with pytest.raises(ValueError, match='riemann'):
    batch.BatchStepper([members[0], (cfg, other[1])])
