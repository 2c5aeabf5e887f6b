"""Conserved-state files for output and restarts.

The reference hands file I/O to the swirl_lm driver: `start_step` and the
`states_to_file` / `states_from_file` options of its configuration
(parameter.py:46-49, 74) and the zero-filling initializer used before a
restart load (initializer.py:41-70). Here one file per field, replica and
step is written in NumPy's `.npy` format: the full halo-padded array in the
storage layout [z, x, y] with the stored dtype, so that a run restarts from
exactly the state it wrote. A second small file per replica and step holds
the simulation time.

  {prefix}-field-{name}-xyz-{cx}-{cy}-{cz}-step-{step}.npy
  {prefix}-time-xyz-{cx}-{cy}-{cz}-step-{step}.npy

Writes go to a temporary name first and are renamed into place, so a file
that exists is complete.
"""

import os
from typing import Dict, Iterable, Optional, Sequence, Tuple

import numpy as np
import torch


def field_path(prefix: str, name: str, coordinate: Sequence[int],
               step: int) -> str:
  cx, cy, cz = (int(c) for c in coordinate)
  return f'{prefix}-field-{name}-xyz-{cx}-{cy}-{cz}-step-{int(step)}.npy'


def time_path(prefix: str, coordinate: Sequence[int], step: int) -> str:
  cx, cy, cz = (int(c) for c in coordinate)
  return f'{prefix}-time-xyz-{cx}-{cy}-{cz}-step-{int(step)}.npy'


def _save_npy(path: str, arr: np.ndarray) -> None:
  tmp = f'{path}.tmp{os.getpid()}'
  with open(tmp, 'wb') as f:
    np.save(f, arr)
  os.replace(tmp, path)


def save_state(prefix: str, state: Dict[str, torch.Tensor], step: int,
               coordinate: Sequence[int] = (0, 0, 0),
               names: Optional[Iterable[str]] = None,
               t: Optional[float] = None) -> None:
  """Writes `state[name]` for each name (all keys by default) at `step`,
  and the time `t` when given. Device tensors are copied to the host first
  (one copy per field)."""
  out_dir, _ = os.path.split(prefix)
  if out_dir:
    os.makedirs(out_dir, exist_ok=True)
  names = list(state) if names is None else list(names)
  for name in names:
    if name not in state:
      raise KeyError(f'{name} is not in the state.')
    arr = state[name].detach().to('cpu').contiguous().numpy()
    _save_npy(field_path(prefix, name, coordinate, step), arr)
  if t is not None:
    _save_npy(time_path(prefix, coordinate, step),
              np.asarray([float(t)], np.float64))


def load_state(prefix: str, names: Iterable[str], step: int,
               coordinate: Sequence[int] = (0, 0, 0),
               device=None, dtype: Optional[torch.dtype] = None
               ) -> Tuple[Dict[str, torch.Tensor], Optional[float]]:
  """Reads the fields `names` written at `step`; returns them (on `device`,
  converted to `dtype` when given) and the time of that step, or None when
  no time was written. All fields must have the same shape."""
  out: Dict[str, torch.Tensor] = {}
  shape = None
  for name in names:
    path = field_path(prefix, name, coordinate, step)
    if not os.path.exists(path):
      raise FileNotFoundError(f'No state file {path}.')
    arr = np.load(path, allow_pickle=False)
    if arr.ndim != 3:
      raise ValueError(f'{path} holds a {arr.ndim}-D array; fields are 3-D.')
    if shape is None:
      shape = arr.shape
    elif arr.shape != shape:
      raise ValueError(f'{path} has shape {arr.shape}, other fields '
                       f'{shape}.')
    t = torch.from_numpy(arr)
    if dtype is not None:
      t = t.to(dtype)
    out[name] = t.to(device) if device is not None else t
  tp = time_path(prefix, coordinate, step)
  time = float(np.load(tp, allow_pickle=False)[0]) if os.path.exists(tp) \
      else None
  return out, time
