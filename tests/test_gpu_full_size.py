"""GPU: parity at the benchmark sizes.

* Kelvin-Helmholtz 256^3: one CFL step of the fused float32 path against the
  float32 oracle over every z-slab of the grid (tests/slab_oracle.py, host
  processes), bar 1e-5 relative L2 per conserved field (or 2x the float32
  noise floor of a field, measured as the oracle's float32 result against
  the float64 build of the kernels); then 100 steps of the float32 path
  against the same kernels in float64 on the float64 run's dt sequence,
  bar 1e-3 (2e-3 for rho_w, the seeded +-1e-3 noise field).
* Buoyant bubble 512x512x256: the same one-step comparison on four z-slabs
  (bottom wall, the bubble, mid-height, top wall), with and without the
  reference's hydrostatic helper states p_ref / rho_ref
  (demo/buoyant_bubble/buoyant_bubble.py:321-323); then 50 steps in
  float32 against float64, both ways. Without the helper states the
  horizontal momentum (|rho u| <= 3e-4 against a 1e5 Pa hydrostatic
  balance whose float32 ulp is ~0.01) is float32 rounding noise after 50
  steps, so only rho and rho_e are held to 1e-3 there. The helper states
  cut that error about fivefold (0.93 to 0.18 measured) but do not make
  the horizontal momentum accurate in float32.
"""

import numpy as np
import pytest
import torch

from oracle import swirlc_oracle as orc
from tests import slab_oracle

pytestmark = pytest.mark.gpu
NAMES = orc.BASE_CONSERVATIVE
KEYS = ('halo_width', 'dx', 'dy', 'dz', 'interpolation_scheme',
        'numeric_flux_scheme', 'include_diffusion', 'transport_parameters',
        'muscl_limiter', 'x', 'y', 'z', 'bc', 'g', 'source_functions',
        'time_integration_scheme')


def _stepper(user_cfg, state, dtype, helper=None, dt=None):
  from swirlc_b200 import engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  cfg = parameter.SwirlCParameters(user_cfg)
  f = [torch.tensor(state[k], dtype=dtype, device='cuda') for k in NAMES]
  s = engine.Solver(cfg, physics_models.PhysicsModels(cfg), f[0].shape, dtype)
  hp = None
  if helper:
    hp = {k: torch.tensor(v, dtype=dtype, device='cuda')
          for k, v in helper.items()}
  if dt is None:
    return engine.Stepper(s, f, dt=cfg.dt, cfl=cfg.cfl, helper=hp)
  return engine.Stepper(s, f, dt=dt, helper=hp)


def _windows(fields, slabs, hw):
  return [{k: v[z0 + hw:z1 + hw, hw:-hw, hw:-hw].double().cpu().numpy()
           for k, v in zip(NAMES, fields)} for z0, z1 in slabs]


def _cat(wins, k):
  return np.concatenate([w[k].astype(np.float64).ravel() for w in wins])


def _rel(a, b):
  n = np.linalg.norm(b)
  return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def _one_step_vs_oracle(user_cfg, state, slabs, helper=None):
  """GPU float32 CFL step against the oracle (float32) on the slabs, with
  the oracle's own dt; the noise floor from the float64 build of the
  kernels. Returns {field: (error, floor)}."""
  hw = user_cfg['halo_width']
  ocfg = orc.make_cfg(**{k: user_cfg[k] for k in KEYS if k in user_cfg})
  s32 = {k: v.astype(np.float32) for k, v in state.items()}
  dt = float(user_cfg['cfl']) * orc.cfl_dt_min(s32, ocfg)
  st = _stepper(user_cfg, state, torch.float32, helper)
  st.step(1)
  gpu_dt = float(st.clock[1].item())
  assert abs(gpu_dt - dt) <= 1e-6 * dt, (gpu_dt, dt)
  g32 = _windows(st.u, slabs, hw)
  del st
  st = _stepper(user_cfg, state, torch.float64, helper, dt=dt)
  st.step(1)
  g64 = _windows(st.u, slabs, hw)
  del st
  torch.cuda.empty_cache()
  want = slab_oracle.one_step(ocfg, state, dt, slabs, np.float32, helper)
  return {k: (_rel(_cat(g32, k), _cat(want, k)),
              _rel(_cat(want, k), _cat(g64, k))) for k in NAMES}


def _f32_vs_f64(user_cfg, state, steps, helper=None):
  """float32 run on the float64 run's dt sequence; rel L2 per field."""
  hw = user_cfg['halo_width']
  st = _stepper(user_cfg, state, torch.float64, helper)
  dts = []
  for _ in range(steps):
    st.step(1)
    dts.append(float(st.clock[1].item()))
  sl = (slice(hw, -hw),) * 3
  f64 = [x[sl].clone() for x in st.u]
  del st
  torch.cuda.empty_cache()
  st = _stepper(user_cfg, state, torch.float32, helper, dt=dts[0])
  for dt in dts:
    st.clock[1] = dt
    st.step(1)
  err = {}
  for k, a, b in zip(NAMES, st.u, f64):
    d = torch.linalg.vector_norm(a[sl].double() - b)
    n = torch.linalg.vector_norm(b)
    err[k] = float(d / n) if float(n) > 0 else float(d)
  return err


def test_kelvin_helmholtz_256_one_step_matches_oracle():
  from swirlc_b200 import configs
  user_cfg, state = configs.kelvin_helmholtz(n=256)
  slabs = [(z, z + 16) for z in range(0, 256, 16)]
  res = _one_step_vs_oracle(user_cfg, state, slabs)
  print('kh256 one step (err, f32 floor):', res)
  for k, (err, floor) in res.items():
    assert err <= max(1e-5, 2.0 * floor), (k, err, floor)


def test_kelvin_helmholtz_256_100_steps_float32_vs_float64():
  from swirlc_b200 import configs
  user_cfg, state = configs.kelvin_helmholtz(n=256)
  err = _f32_vs_f64(user_cfg, state, 100)
  print('kh256 100 steps f32 vs f64:', err)
  for k, e in err.items():
    # rho_w is the seeded +-1e-3 noise field: its float32 rounding grows to
    # 1.3e-3 of its own norm in 100 steps (the other fields stay <= 2e-5).
    assert e <= (2e-3 if k == 'rho_w' else 1e-3), (k, e)


BUBBLE_SLABS = [(0, 16), (70, 86), (120, 136), (240, 256)]


@pytest.mark.parametrize('with_helper', [False, True],
                         ids=['plain', 'p_ref_rho_ref'])
def test_buoyant_bubble_full_size_one_step_matches_oracle(with_helper):
  from swirlc_b200 import configs
  user_cfg, state = configs.buoyant_bubble()
  helper = configs.buoyant_bubble_reference_states() if with_helper else None
  res = _one_step_vs_oracle(user_cfg, state, BUBBLE_SLABS, helper)
  print('bubble one step (err, f32 floor):', with_helper, res)
  for k, (err, floor) in res.items():
    assert err <= max(1e-5, 2.0 * floor), (k, err, floor)


def test_buoyant_bubble_full_size_50_steps_float32_vs_float64():
  from swirlc_b200 import configs
  user_cfg, state = configs.buoyant_bubble()
  plain = _f32_vs_f64(user_cfg, state, 50)
  helped = _f32_vs_f64(user_cfg, state, 50,
                       configs.buoyant_bubble_reference_states())
  print('bubble 50 steps f32 vs f64, plain:', plain)
  print('bubble 50 steps f32 vs f64, p_ref/rho_ref:', helped)
  for k in ('rho', 'rho_e'):
    assert plain[k] <= 1e-3, (k, plain[k])
    assert helped[k] <= 1e-3, (k, helped[k])
  for k in ('rho_u', 'rho_v'):
    assert helped[k] <= 0.25 * plain[k], (k, helped[k], plain[k])
