"""Float32 error of each benchmark set-up against the same kernels in float64.

  python -m swirlc_b200.accuracy [--configs sod,kh,bubble] [--small]

Runs the fused CUDA path twice from the same seeded initial state, in float32
and float64, with the float64 run's dt sequence replayed in float32 (fixed dt
per step), and prints one JSON line per config with the relative L2 error per
conserved field on interior cells.
"""

import argparse
import json

import numpy as np
import torch

from swirlc_b200 import configs, engine
from swirlc_b200.common import types
from swirlc_b200.core import parameter
from swirlc_b200.physics import physics_models

NAMES = types.BASE_CONSERVATIVE


def _run(user_cfg, state, steps, dtype, dts=None):
  cfg = parameter.SwirlCParameters(user_cfg)
  pm = physics_models.PhysicsModels(cfg)
  f = [torch.tensor(state[k], dtype=dtype, device='cuda') for k in NAMES]
  s = engine.Solver(cfg, pm, f[0].shape, dtype)
  if dts is None:
    st = engine.Stepper(s, f, dt=cfg.dt, cfl=cfg.cfl, t_end=cfg.t_end,
                        scheme=cfg.time_integration_scheme)
    out = []
    for _ in range(steps):
      st.step(1)
      out.append(float(st.clock[1].item()))
      if cfg.t_end > 0 and st.time() >= cfg.t_end - 1e-12:
        break
    return f, out
  st = engine.Stepper(s, f, dt=0.0, scheme=cfg.time_integration_scheme)
  for dt in dts:
    st.clock[1] = dt
    st.step(1)
  return f, dts


def report(name, user_cfg, state, steps):
  f64, dts = _run(user_cfg, state, steps, torch.float64)
  f32, _ = _run(user_cfg, state, steps, torch.float32, dts)
  hw = user_cfg['halo_width']
  sl = (slice(hw, -hw),) * 3
  err = {}
  for k, a, b in zip(NAMES, f32, f64):
    a = a.double()[sl]
    b = b[sl]
    den = float(torch.linalg.vector_norm(b))
    err[k] = float(torch.linalg.vector_norm(a - b)) / (den if den else 1.0)
  return {'config': name, 'steps': len(dts), 't': float(np.sum(dts)),
          'rel_l2_f32_vs_f64': err}


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--configs', default='sod,kh,bubble')
  ap.add_argument('--small', action='store_true')
  a = ap.parse_args()
  for name in a.configs.split(','):
    if name == 'sod':
      user_cfg, state = configs.sod()
      steps = 10000
    elif name == 'kh':
      user_cfg, state = configs.kelvin_helmholtz(n=64 if a.small else 256)
      steps = 100
    elif name == 'bubble':
      user_cfg, state = (configs.buoyant_bubble(64, 64, 32) if a.small else
                         configs.buoyant_bubble())
      steps = 50
    else:
      raise ValueError(name)
    print(json.dumps(report(name, user_cfg, state, steps)), flush=True)


if __name__ == '__main__':
  main()
