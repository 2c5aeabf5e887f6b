"""Helper functions (reference: common/utils.py:24-216).

Mesh helpers run on the host in NumPy (they build the small 1-D coordinate
arrays the kernels read); the conversions run on the tensors' device.
"""

from typing import Dict, Sequence

import numpy as np
import torch

from swirlc_b200.common import types


def mesh_local_size(cfg) -> list:
  """utils.py:24-40."""
  n_core = [cfg.cx, cfg.cy, cfg.cz]
  n = [np.asarray(cfg.x).shape[0], np.asarray(cfg.y).shape[0],
       np.asarray(cfg.z).shape[0]]
  return [int(n_i / c) for n_i, c in zip(n, n_core)]


def mesh_local(replica_id, replicas: np.ndarray, cfg,
               dtype=np.float32) -> Dict[str, np.ndarray]:
  """utils.py:43-89, including its halo-coordinate rule: the low halo is
  `dx * [-hw, ..., -1]` (utils.py:68), not `x[0] - dx * [hw, ..., 1]`."""
  n_local = mesh_local_size(cfg)
  core_idx = np.argwhere(np.asarray(replicas) == int(replica_id))[0]
  hw = cfg.halo_width
  out = {}
  for i, dim in enumerate(types.DIMS):
    m = np.asarray(getattr(cfg, dim), dtype=dtype)
    halo_lo = np.linspace(-hw, -1, hw).astype(dtype)
    halo_hi = np.linspace(1, hw, hw).astype(dtype)
    full = np.concatenate([(m[1] - m[0]) * halo_lo, m,
                           m[-1] + (m[-1] - m[-2]) * halo_hi])
    idx = np.linspace(core_idx[i] * n_local[i],
                      (core_idx[i] + 1) * n_local[i] + 2 * hw - 1,
                      n_local[i] + 2 * hw).astype(np.int32)
    out[dim] = full[idx]
  return out


def gravity_direction(cfg) -> int:
  """utils.py:114-142: -1 none, 0/1/2 aligned axis, 3 misaligned."""
  g_vec = np.fromiter((cfg.g[dim] for dim in types.DIMS), dtype=float)
  if np.abs(np.linalg.norm(g_vec) - 1.0) >= types.SMALL:
    return -1
  g_dim = 3
  for i in range(len(types.DIMS)):
    if np.abs(np.abs(cfg.g[types.DIMS[i]]) - 1.0) < types.SMALL:
      g_dim = i
      break
  return g_dim


def conservative_to_primitive_variables(states):
  """utils.py:145-183."""
  inv_rho = 1.0 / states[types.RHO]
  prim = {types.RHO: states[types.RHO]}
  for key, val in states.items():
    if key == types.RHO:
      continue
    if types.is_conservative_name(key):
      prim[types.conservative_to_primitive_name(key)] = inv_rho * val
  return prim


def primitive_to_conservative_variables(states):
  """utils.py:186-216."""
  out = {}
  for key, val in states.items():
    if key == types.RHO:
      out[types.RHO] = states[types.RHO]
    else:
      out[types.primitive_to_conservative_name(key)] = states[types.RHO] * val
  return out


def as_tensor3d(f) -> torch.Tensor:
  """A FlowFieldVar (3-D tensor or list of nz 2-D slices) as a 3-D tensor."""
  if isinstance(f, torch.Tensor):
    return f
  if isinstance(f, (list, tuple)):
    return torch.stack([torch.as_tensor(x) for x in f])
  return torch.as_tensor(np.asarray(f))


def like_input(t: torch.Tensor, ref):
  """Returns `t` in the representation of `ref` (tensor or list of slices)."""
  if isinstance(ref, (list, tuple)):
    return list(torch.unbind(t, 0))
  return t
