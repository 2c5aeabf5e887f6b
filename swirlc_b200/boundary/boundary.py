"""Boundary conditions (reference: boundary/boundary.py).

`exchange_halos`, `update_boundary` and `update_conservative_cell_averages`
fill halos with the swc_halo_fill kernel: dims in order x, y, z, PERIODIC
wrap, DIRICHLET scalar or per-layer planes, NEUMANN layer-by-layer
extrapolation, and BCs given on a primitive applied to field/rho and
multiplied back by the updated rho (boundary.py:34-86, 464-539, 606-629).
With more than one replica (the grid split into cx x cy x cz blocks, one
per process, rank = replica id), sides shared with another replica receive
its interior layers through `halo_exchange.DistExchange` (torch.distributed),
dim by dim; per-layer Dirichlet planes are then given per replica, as the
reference expects them.
"""

import ctypes
from typing import Dict

import numpy as np
import torch

from swirlc_b200 import _native as nat
from swirlc_b200 import engine
from swirlc_b200.boundary import bc_types
from swirlc_b200.common import types
from swirlc_b200.common import utils

_CELL_AVG_BC = bc_types.BoundaryDictionaryType.CELL_AVERAGES.value


def _grid_for(t: torch.Tensor, width: int) -> nat.SwcGrid:
  nza, nxa, nya = t.shape
  g = nat.SwcGrid(nxa - 2 * width, nya - 2 * width, nza - 2 * width, width,
                  nya, nya * nxa, 1.0, 1.0, 1.0)
  if min(g.nx, g.ny, g.nz) <= 0:
    raise ValueError(f'Shape {tuple(t.shape)} too small for width {width}.')
  return g


def _fill(fields, specs, vias, width: int, rho_index: int = -1):
  t0 = fields[0]
  grid = _grid_for(t0, width)
  arr = (nat.SwcFieldBC * len(fields))()
  keep = []
  for i, (spec, via) in enumerate(zip(specs, vias)):
    keep += engine.fill_field_bc(arr[i], spec, via, t0.shape, width, t0.dtype,
                                 t0.device)
  nat.check(nat.load().swc_halo_fill(
      ctypes.byref(grid), nat.dtype_code(t0.dtype), len(fields),
      nat.ptr_array(fields), arr, rho_index, nat.stream_ptr()), 'halo fill')
  del keep


def _periodic_of(specs):
  out = []
  for d in types.DIMS:
    kinds = {bool(spec and spec.get(d)) and any(
        bc_types.bc_value(v[0]) == 0 for v in spec[d].values())
             for spec in specs}
    if len(kinds) != 1:
      raise NotImplementedError(
          f'Fields disagree on whether dim {d} is periodic across replicas.')
    out.append(kinds.pop())
  return out


def _fill_replicas(replica_id, replicas, fields, specs, vias, width: int):
  """Halo update of `fields` (rho first when any BC is on a primitive) of
  this replica: BCs on its outer sides, neighbours' layers on the others."""
  from swirlc_b200 import halo_exchange as hx
  import types as pytypes
  t0 = fields[0]
  grid = _grid_for(t0, width)
  arr = (nat.SwcFieldBC * len(fields))()
  keep = []
  for i, (spec, via) in enumerate(zip(specs, vias)):
    keep += engine.fill_field_bc(arr[i], spec, via, t0.shape, width, t0.dtype,
                                 t0.device)
  layout = hx.BlockLayout(np.asarray(replicas), _periodic_of(specs))
  masked = hx.masked_bcs(pytypes.SimpleNamespace(bcs=arr), layout,
                         int(replica_id), nat)

  def bc_fill(rid, fs, dim):
    nat.check(nat.load().swc_halo_fill(
        ctypes.byref(grid), nat.dtype_code(t0.dtype), len(fs),
        nat.ptr_array(fs), masked[dim], 0, nat.stream_ptr()), 'halo fill')

  hx.DistExchange(layout, width, bc_fill, vias).fill([fields],
                                                     [int(replica_id)])
  del keep


def exchange_halos(replica_id, replicas, u, bc_dict, width: int):
  """boundary.py:34-86 for one field; returns a new, halo-filled field."""
  t = utils.as_tensor3d(u).contiguous().clone()
  if width > 0:
    if np.asarray(replicas).size != 1:
      _fill_replicas(replica_id, replicas, [t], [bc_dict], [0], width)
    else:
      _fill([t], [bc_dict], [0], width)
  return utils.like_input(t, u)


def update_boundary(replica_id, replicas, states: Dict, cfg) -> Dict:
  """boundary.py:606-629."""
  return {k: exchange_halos(replica_id, replicas, v, cfg.bc[k], cfg.halo_width)
          for k, v in states.items()}


def update_conservative_cell_averages(replica_id, replicas, conservative,
                                      cfg) -> Dict:
  """boundary.py:464-539: halo fill of every conserved variable."""
  bc = cfg.bc[_CELL_AVG_BC]
  names = list(conservative.keys())
  specs, vias = [], []
  for name in names:
    prim = types.conservative_to_primitive_name(name)
    if name in bc:
      specs.append(bc[name]); vias.append(0)
    elif prim in bc:
      specs.append(bc[prim]); vias.append(1)
    else:
      raise ValueError(
          'A "cells" boundary condition is required for all conservative'
          ' variables, either directly or through their respective primitive.'
          f' No boundary condition was found for {name} or {prim}.')
  fields = [utils.as_tensor3d(conservative[n]).contiguous().clone()
            for n in names]
  rho_index = names.index(types.RHO) if types.RHO in names else -1
  if any(vias) and rho_index < 0:
    raise ValueError('Primitive boundary conditions need rho.')
  # rho first so primitive BCs see its final halos (boundary.py:484-487).
  order = ([rho_index] if rho_index >= 0 else []) + [
      i for i in range(len(names)) if i != rho_index]
  if cfg.halo_width > 0 and np.asarray(replicas).size != 1:
    if len(order) > nat.SWC_MAX_FIELDS:
      raise NotImplementedError(
          f'At most {nat.SWC_MAX_FIELDS} fields per multi-replica halo update.')
    _fill_replicas(replica_id, replicas, [fields[i] for i in order],
                   [specs[i] for i in order], [vias[i] for i in order],
                   cfg.halo_width)
  elif cfg.halo_width > 0:
    for lo in range(0, len(order), nat.SWC_MAX_FIELDS):
      chunk = order[lo:lo + nat.SWC_MAX_FIELDS]
      if rho_index >= 0 and rho_index not in chunk and any(vias[i] for i in chunk):
        chunk = [rho_index] + chunk
      _fill([fields[i] for i in chunk], [specs[i] for i in chunk],
            [vias[i] for i in chunk], cfg.halo_width,
            chunk.index(rho_index) if rho_index in chunk else -1)
  return {n: utils.like_input(fields[i], conservative[n])
          for i, n in enumerate(names)}
