"""Step loop (reference: core/driver.py:202-226, which runs the swirl_lm
driver: init_fn per replica, then num_cycles x num_steps Simulation.step).

`solver(init_fn, cfg)` builds the initial state with `init_fn(replica_id,
coordinates, cfg)` on the host, moves it to the current CUDA device and
advances it num_cycles x num_steps steps in place with the fused stage
kernels, one step captured in a CUDA graph and replayed. With cfg.cfl > 0
the step size is the device-side CFL reduction, clamped to end at cfg.t_end
when that is > 0; otherwise cfg.dt. `on_cycle(cycle, state, t)` is called
after every cycle (e.g. to write the states out). Single replica; the
domain-decomposed loop is swirlc_b200.parallel.
"""

from typing import Callable, Dict, Optional

import numpy as np
import torch

from swirlc_b200 import engine
from swirlc_b200.common import types
from swirlc_b200.common import utils
from swirlc_b200.physics import physics_models as physics_models_lib


def run(state: Dict[str, torch.Tensor], cfg, steps: int,
        physics_models=None, graph: bool = True,
        on_step: Optional[Callable] = None) -> engine.Stepper:
  """Advances `state` (CUDA tensors, reference layout) in place by `steps`
  steps; returns the Stepper (its clock holds t and the step count)."""
  pm = physics_models or physics_models_lib.PhysicsModels(cfg)
  fields = [utils.as_tensor3d(state[k]).contiguous()
            for k in types.BASE_CONSERVATIVE]
  for k, f in zip(types.BASE_CONSERVATIVE, fields):
    state[k] = f
  solver = engine.Solver(cfg, pm, fields[0].shape, fields[0].dtype,
                         fields[0].device)
  stepper = engine.Stepper(solver, fields, dt=cfg.dt,
                           cfl=float(getattr(cfg, 'cfl', 0.0) or 0.0),
                           t_end=float(getattr(cfg, 't_end', 0.0) or 0.0),
                           scheme=cfg.time_integration_scheme)
  if steps <= 0:
    return stepper
  done = 0
  if graph and on_step is None and steps > 1:
    stepper.step(1)
    stepper.capture()
    done = 1
  while done < steps:
    stepper.step(1)
    done += 1
    if on_step is not None:
      on_step(stepper)
  return stepper


def solver(customized_init_fn, cfg, on_cycle: Optional[Callable] = None,
           dtype=torch.float32):
  """driver.py:202-226: runs the simulation; returns the final state dict."""
  if cfg.cx * cfg.cy * cfg.cz != 1:
    raise NotImplementedError(
        'Multi-replica runs go through swirlc_b200.parallel.')
  init = customized_init_fn(0, (0, 0, 0), cfg)
  dev = torch.device('cuda', torch.cuda.current_device())
  state = {k: utils.as_tensor3d(init[k]).to(device=dev, dtype=dtype)
           .contiguous() for k in types.BASE_CONSERVATIVE}
  stepper = run(state, cfg, 0)
  for cycle in range(cfg.num_cycles):
    if stepper.graph is None and cfg.num_steps > 1:
      stepper.step(1)
      stepper.capture()
      stepper.step(cfg.num_steps - 1)
    else:
      stepper.step(cfg.num_steps)
    if on_cycle is not None:
      torch.cuda.synchronize()
      on_cycle(cycle, state, stepper.time())
  torch.cuda.synchronize()
  return state
