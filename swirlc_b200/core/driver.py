"""Step loop (reference: core/driver.py:202-226, which runs the swirl_lm
driver: init_fn per replica, then num_cycles x num_steps Simulation.step).

`solver(init_fn, cfg)` builds the initial state with `init_fn(replica_id,
coordinates, cfg)` on the host, moves it to the current CUDA device and
advances it num_cycles x num_steps steps in place with the fused stage
kernels, one step captured in a CUDA graph and replayed. With cfg.cfl > 0
the step size is the device-side CFL reduction, clamped to end at cfg.t_end
when that is > 0; otherwise cfg.dt. `on_cycle(cycle, state, t)` is called
after every cycle. With `dump_prefix` the configuration is saved as YAML
and the conserved state (with the time) is written after every cycle at step
start_step + (cycle + 1) * num_steps; with `load_prefix` the run restarts
from the state written at cfg.start_step instead of calling the initializer
(swirlc_b200.core.state_io gives the file layout). Single replica; the
domain-decomposed loop is swirlc_b200.decomposition.
"""

from typing import Callable, Dict, Optional

import numpy as np
import torch

from swirlc_b200 import engine
from swirlc_b200.common import types
from swirlc_b200.common import utils
from swirlc_b200.core import state_io
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
           dtype=torch.float32, dump_prefix: Optional[str] = None,
           load_prefix: Optional[str] = None):
  """driver.py:202-226: runs the simulation; returns the final state dict."""
  if cfg.cx * cfg.cy * cfg.cz != 1:
    raise NotImplementedError(
        'Multi-replica runs go through swirlc_b200.decomposition.')
  dev = torch.device('cuda', torch.cuda.current_device())
  start = int(getattr(cfg, 'start_step', 0) or 0)
  t0 = None
  if load_prefix is not None:
    init, t0 = state_io.load_state(load_prefix, types.BASE_CONSERVATIVE,
                                   start, device=dev, dtype=dtype)
  else:
    init = customized_init_fn(0, (0, 0, 0), cfg)
  state = {k: utils.as_tensor3d(init[k]).to(device=dev, dtype=dtype)
           .contiguous() for k in types.BASE_CONSERVATIVE}
  stepper = run(state, cfg, 0)
  if load_prefix is not None:
    stepper.set_time(t0 if t0 is not None else start * float(cfg.dt), start)
  if dump_prefix is not None:
    cfg.save_to_file(dump_prefix)
  for cycle in range(cfg.num_cycles):
    if stepper.graph is None and cfg.num_steps > 1:
      stepper.step(1)
      stepper.capture()
      stepper.step(cfg.num_steps - 1)
    else:
      stepper.step(cfg.num_steps)
    if dump_prefix is not None:
      torch.cuda.synchronize()
      state_io.save_state(dump_prefix, state,
                          start + (cycle + 1) * cfg.num_steps,
                          names=types.BASE_CONSERVATIVE, t=stepper.time())
    if on_cycle is not None:
      torch.cuda.synchronize()
      on_cycle(cycle, state, stepper.time())
  torch.cuda.synchronize()
  return state
