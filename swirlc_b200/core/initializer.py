"""Initial-condition layout (reference: core/initializer.py:23-322).

`partial_field_for_core` evaluates a value function on the local mesh of a
core (cell centres from cfg.x/y/z, order x, y, z), pads the halo with the
given mode and permutes to the storage layout [z, x, y]. Value functions
receive NumPy arrays; the result is a float32 (or `dtype`) torch tensor on
`device` (CPU by default, to be moved where the solver runs).
"""

from typing import Callable, Dict, Optional, Sequence

import numpy as np
import torch

_DEFAULT_PERMUTATION = (2, 0, 1)
_PAD = {'SYMMETRIC': 'symmetric', 'REFLECT': 'reflect', 'CONSTANT': 'constant'}

ValueFunction = Callable[..., np.ndarray]


def _local_1d_mesh(core_n: int, core_id: int, global_1d_mesh) -> np.ndarray:
  """initializer.py:226-253."""
  m = np.asarray(global_1d_mesh)
  idx = np.linspace(core_id * core_n, (core_id + 1) * core_n - 1,
                    core_n).astype(np.int32)
  return m[idx]


def partial_field_for_core(cfg, coordinate: Sequence[int],
                           value_fn: ValueFunction,
                           perm: Optional[Sequence[int]] = _DEFAULT_PERMUTATION,
                           pad_mode: Optional[str] = 'SYMMETRIC',
                           dtype=torch.float32,
                           device=None) -> torch.Tensor:
  """initializer.py:73-223."""
  gx, gy, gz = (int(c) for c in coordinate)
  for g, c, name in ((gx, cfg.cx, 'x'), (gy, cfg.cy, 'y'), (gz, cfg.cz, 'z')):
    if g < 0 or g >= c:
      raise ValueError(f'Invalid subgrid coordinate specified with {name} '
                       'core index.')
  for n, name in ((cfg.core_nx, 'core_nx'), (cfg.core_ny, 'core_ny'),
                  (cfg.core_nz, 'core_nz')):
    if n < cfg.halo_width:
      raise ValueError(f'Local mesh size `{name} = {n}` must be at least the '
                       f'halo width `cfg.halo_width = {cfg.halo_width}`.')
  xs = _local_1d_mesh(cfg.core_nx, gx, cfg.x)
  ys = _local_1d_mesh(cfg.core_ny, gy, cfg.y)
  zs = _local_1d_mesh(cfg.core_nz, gz, cfg.z)
  xx, yy, zz = np.meshgrid(xs, ys, zs, indexing='ij')
  val = np.asarray(value_fn(xx, yy, zz, np.float32(cfg.lx), np.float32(cfg.ly),
                            np.float32(cfg.lz), coordinate))
  val = np.broadcast_to(val, xx.shape)
  if pad_mode:
    if pad_mode not in _PAD:
      raise ValueError(f'Unknown pad mode {pad_mode}.')
    hw = cfg.halo_width
    val = np.pad(val, [(hw, hw)] * 3, mode=_PAD[pad_mode])
  if perm:
    val = np.transpose(val, perm)
  return torch.tensor(np.ascontiguousarray(val), dtype=dtype, device=device)


def default_initializer(replica_id, coordinates, cfg) -> Dict[str, torch.Tensor]:
  """initializer.py:41-70: zeros for every conservative variable."""
  del replica_id
  return {name: partial_field_for_core(cfg, coordinates,
                                       constant_initial_state_fn(0.0))
          for name in cfg.conservative_variable_names}


def constant_initial_state_fn(value: float) -> ValueFunction:
  """initializer.py:257-274."""

  def init_fn(xx, yy, zz, lx, ly, lz, coord):
    del yy, zz, lx, ly, lz, coord
    return value * np.ones_like(xx)

  return init_fn


def step_function_initial_state_fn(left_value: float, right_value: float,
                                   step_loc: float, dim: str) -> ValueFunction:
  """initializer.py:277-322: left_value where |coord / L| <= step_loc."""

  def init_fn(xx, yy, zz, lx, ly, lz, coord):
    del coord
    v, l = {'x': (xx, lx), 'y': (yy, ly), 'z': (zz, lz)}[dim]
    return np.where(np.abs(v / l) <= step_loc, left_value * np.ones_like(v),
                    right_value * np.ones_like(v))

  return init_fn
