"""GPU: the non-finite detector of the fused CFL reduction.

A non-finite value is injected into the input state on the host (the only
injection route: no kernel is made to fault). The step's fused CFL
reduction then reports it through the device clock, and
`Stepper.step(check=True)` / `BatchStepper.step(check=True)` raise
FloatingPointError (C status SWC_ERR_NONFINITE from swc_clock_status).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
NAMES = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')


def _stepper(n=16, cfl=0.5, inject=None, dtype=torch.float32):
  from swirlc_b200 import configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  user_cfg, state = configs.kelvin_helmholtz(n=n, nu=1e-3)
  cfg = parameter.SwirlCParameters(user_cfg)
  state = {k: v.copy() for k, v in state.items()}
  if inject is not None:
    name, value = inject
    state[name][7, 5, 9] = value  # an interior cell (halo width 3)
  f = [torch.tensor(state[k], dtype=dtype, device='cuda') for k in NAMES]
  s = engine.Solver(cfg, physics_models.PhysicsModels(cfg), f[0].shape, dtype)
  return engine.Stepper(s, f, dt=1e-3, cfl=cfl)


@pytest.mark.parametrize('dtype', [torch.float32, torch.float64])
@pytest.mark.parametrize('cfl', [0.5, 0.0])
def test_clean_state_passes_the_check(cfl, dtype):
  st = _stepper(cfl=cfl, dtype=dtype)
  st.step(3, check=True)
  assert st.steps_done() == 3


@pytest.mark.parametrize('inject', [('rho_e', float('nan')),
                                    ('rho', float('inf')),
                                    ('rho_u', float('-inf')),
                                    ('rho_e', -5.0)],  # p < 0
                         ids=['nan_rho_e', 'inf_rho', 'ninf_rho_u', 'neg_p'])
@pytest.mark.parametrize('cfl', [0.5, 0.0])
def test_injected_bad_state_is_reported(inject, cfl):
  st = _stepper(cfl=cfl, inject=inject)
  with pytest.raises(FloatingPointError, match='non-finite or unphysical'):
    st.step(1, check=True)
  # Graph replays report it the same way.
  st2 = _stepper(cfl=cfl, inject=inject)
  st2.step(1)
  st2.capture()
  with pytest.raises(FloatingPointError):
    st2.step(2, check=True)


def test_cfl_reduce_flags_a_bad_initial_state():
  from swirlc_b200 import _native as nat
  st = _stepper(cfl=0.0, inject=('rho_e', float('nan')))
  out = torch.full((1,), 1e300, dtype=torch.float64, device='cuda')
  st.s.cfl_reduce(st.u, out)
  assert float(out.item()) == 0.0
  clock = torch.zeros(6, dtype=torch.float64, device='cuda')
  clock[2] = 0.0
  with pytest.raises(FloatingPointError):
    nat.check(nat.load().swc_clock_status(clock.data_ptr(), nat.stream_ptr()))
  clock[2] = 1e-3
  nat.check(nat.load().swc_clock_status(clock.data_ptr(), nat.stream_ptr()))
  with pytest.raises(ValueError):
    nat.check(nat.load().swc_clock_status(None, nat.stream_ptr()))


def test_batch_names_the_bad_member():
  from swirlc_b200 import batch, configs
  members = configs.riemann_batch(members=3, seed=1)
  members[1][1]['rho_e'][4, 6, 4] = np.nan
  b = batch.BatchStepper(members)
  with pytest.raises(FloatingPointError, match='batch member 1'):
    b.step(1, check=True)
  good = configs.riemann_batch(members=3, seed=1)
  batch.BatchStepper(good).step(2, check=True)
