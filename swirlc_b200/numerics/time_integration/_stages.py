"""Stage algebra shared by rk3 and rk2 for user-supplied rhs functions."""

import torch

from swirlc_b200 import _native as nat
from swirlc_b200.common import utils


def combine(mode, c0, c1, dt_t, u0, uk, l):
  """Elementwise RK combination on the device (swc_rk_combine)."""
  ukt = utils.as_tensor3d(uk).contiguous()
  lt = utils.as_tensor3d(l).to(ukt.dtype).contiguous()
  u0t = None if u0 is None else utils.as_tensor3d(u0).contiguous()
  if not ukt.is_cuda:
    raise ValueError('RK stages need CUDA tensors.')
  out = torch.empty_like(ukt)
  lib = nat.load()
  nat.check(lib.swc_rk_combine(
      ukt.numel(), nat.dtype_code(ukt.dtype), mode, float(c0), float(c1),
      dt_t.data_ptr(), None if u0t is None else u0t.data_ptr(),
      ukt.data_ptr(), lt.data_ptr(), out.data_ptr(), nat.stream_ptr()),
      'rk combine')
  return utils.like_input(out, uk)


def dt_tensor(dt, device):
  return torch.tensor([float(dt)], dtype=torch.float64, device=device)


def first_device(state):
  for v in state.values():
    t = utils.as_tensor3d(v)
    return t.device
  raise ValueError('Empty state.')
