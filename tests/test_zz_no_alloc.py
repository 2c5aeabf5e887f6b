"""GPU: swc_rk_step_noalloc (work states in the library's built-in device
array) gives the same states as swc_rk_step with caller-supplied work
buffers, bit for bit, over two calls in a row.

Named to be collected after every other test file, so that it also runs in a
process where the other tests have already used the library."""

import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(n, dtype, scheme):
  from swirlc_b200 import configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  user_cfg, state = configs.kelvin_helmholtz(n=n, nu=1e-3)
  user_cfg['time_integration_scheme'] = scheme
  cfg = parameter.SwirlCParameters(user_cfg)
  pm = physics_models.PhysicsModels(cfg)
  f = [torch.tensor(state[k], dtype=dtype, device='cuda')
       for k in ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')]
  return engine.Solver(cfg, pm, f[0].shape, dtype), f


def _clock(dt, cfl):
  c = torch.zeros(6, dtype=torch.float64, device='cuda')
  c[1] = dt
  c[2] = 1e300
  c[3] = cfl
  return c


@pytest.mark.parametrize('scheme,dtype,cfl', [
    ('rk3', torch.float32, 0.0),
    ('rk3', torch.float32, 0.5),
    ('rk2', torch.float64, 0.0),
])
def test_noalloc_step_matches_caller_buffers(scheme, dtype, cfl):
  from swirlc_b200 import _native as nat
  lib = nat.load()
  solver, f = _setup(24, dtype, scheme)
  order = 3 if scheme == 'rk3' else 2
  u_ref = [x.clone() for x in f]
  u_new = [x.clone() for x in f]
  work = [torch.empty_like(x) for x in f for _ in range(2)]
  clock_ref = _clock(2e-3, cfl)
  clock_new = _clock(2e-3, cfl)
  if cfl > 0:
    for c, u in ((clock_ref, u_ref), (clock_new, u_new)):
      solver.fill_halos(u)
      solver.cfl_reduce(u, c[2:3])
  hw = 3
  sl = (slice(hw, -hw),) * 3
  for call in range(2):
    nat.check(lib.swc_rk_step(
        ctypes.byref(solver.grid), ctypes.byref(solver.scheme), solver.bcs,
        order, nat.ptr_array(u_ref), nat.ptr_array(work),
        clock_ref.data_ptr(), nat.stream_ptr()))
    nat.check(lib.swc_rk_step_noalloc(
        ctypes.byref(solver.grid), ctypes.byref(solver.scheme), solver.bcs,
        order, nat.ptr_array(u_new), clock_new.data_ptr(), nat.stream_ptr()))
    torch.cuda.synchronize()
    # The same kernels on the same strides: equal to the bit (a partial
    # overlap of work fields or a stale region of the array would not be).
    for name, a, b in zip(('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e'),
                          u_new, u_ref):
      assert torch.equal(a[sl], b[sl]), (call, name)
    assert torch.equal(clock_new, clock_ref), call
    assert int(clock_new[5:6].view(torch.int64)) == call + 1


def test_noalloc_step_rejects_grid_beyond_scratch():
  from swirlc_b200 import _native as nat
  solver, f = _setup(24, torch.float32, 'rk3')
  big = nat.SwcGrid.from_buffer_copy(solver.grid)
  big.nz = 4000  # 10 fields of 4006 planes of 30*30 floats: 144 MB
  clock = _clock(2e-3, 0.0)
  before = [x.clone() for x in f]
  with pytest.raises(ValueError, match='scratch'):
    nat.check(nat.load().swc_rk_step_noalloc(
        ctypes.byref(big), ctypes.byref(solver.scheme), solver.bcs, 3,
        nat.ptr_array(f), clock.data_ptr(), nat.stream_ptr()))
  torch.cuda.synchronize()
  assert all(torch.equal(a, b) for a, b in zip(f, before))
  assert float(clock[0]) == 0.0
