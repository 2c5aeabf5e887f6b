"""GPU: the one-call time step swc_rk_step (work buffers supplied by the
caller) matches the stage-by-stage composition bit for bit."""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(n=24, dtype=torch.float32, scheme='rk3'):
  from swirlc_b200 import configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  user_cfg, state = configs.kelvin_helmholtz(n=n, nu=1e-3)
  user_cfg['time_integration_scheme'] = scheme
  cfg = parameter.SwirlCParameters(user_cfg)
  pm = physics_models.PhysicsModels(cfg)
  f = [torch.tensor(state[k], dtype=dtype, device='cuda')
       for k in ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')]
  return cfg, engine.Solver(cfg, pm, f[0].shape, dtype), f


@pytest.mark.parametrize('scheme', ['rk3', 'rk2'])
def test_rk_step_matches_stage_composition(scheme):
  from swirlc_b200 import _native as nat
  cfg, solver, f = _setup(scheme=scheme)
  dt = 2e-3
  ref = solver.rk3(f, dt) if scheme == 'rk3' else solver.rk2(f, dt)
  u = [x.clone() for x in f]
  work = [torch.empty_like(x) for x in f for _ in range(2)]
  clock = torch.zeros(6, dtype=torch.float64, device='cuda')
  clock[1] = dt
  clock[2] = 1e300
  nat.check(nat.load().swc_rk_step(
      ctypes.byref(solver.grid), ctypes.byref(solver.scheme), solver.bcs,
      3 if scheme == 'rk3' else 2, nat.ptr_array(u), nat.ptr_array(work),
      clock.data_ptr(), nat.stream_ptr()))
  torch.cuda.synchronize()
  hw = 3
  sl = (slice(hw, -hw),) * 3
  for a, b in zip(u, ref):
    assert torch.equal(a[sl], b[sl])
  assert float(clock[0]) == pytest.approx(dt)
  assert int(clock[5:6].view(torch.int64)) == 1
  assert 0.0 < float(clock[2]) < 1e300  # CFL limit of the new state


def test_rk_step_rejects_bad_arguments():
  from swirlc_b200 import _native as nat
  cfg, solver, f = _setup()
  clock = torch.zeros(6, dtype=torch.float64, device='cuda')
  with pytest.raises(NotImplementedError):
    nat.check(nat.load().swc_rk_step(
        ctypes.byref(solver.grid), ctypes.byref(solver.scheme), solver.bcs, 4,
        nat.ptr_array(f), nat.ptr_array(f + f), clock.data_ptr(),
        nat.stream_ptr()))
  with pytest.raises(ValueError):
    nat.check(nat.load().swc_rk_step(
        ctypes.byref(solver.grid), ctypes.byref(solver.scheme), solver.bcs, 3,
        nat.ptr_array(f), nat.ptr_array(f + f), None, nat.stream_ptr()))
