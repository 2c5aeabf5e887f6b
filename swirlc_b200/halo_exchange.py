"""Halo exchange between the blocks of a decomposed grid.

Replaces swirl_lm `halo_exchange.inplace_halo_exchange` as the reference
calls it from `boundary.exchange_halos` (boundary.py:34-86) when the grid is
split over `replicas` (cx, cy, cz blocks; `replicas[i, j, k]` is the id of the
block at block coordinates (i, j, k), simulation.py:53-56). A block holds its
n/c interior cells per dim plus `halo_width` layers (utils.py:24-40).

Dims are updated in the order x, y, z, each pass covering the full extent of
the other two axes (halos included), so that edges and corners come out as in
the single-grid fill. Along a dim, a side with a neighbouring block (an inner
side, or a periodic wrap when the dim has more than one block) receives the
neighbour's `halo_width` interior layers; the other sides get the physical
boundary condition, or the periodic wrap of a dim that is not split.

Two transports share the slab arithmetic:
  * `DistExchange`: one block per process over `torch.distributed` (NCCL on
    GPUs, gloo on CPUs), paired isend/irecv per dim;
  * `LocalExchange`: every block in this process (copies between blocks);
    used to run a decomposed grid on one device.
"""

import ctypes
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np
import torch

from swirlc_b200.common import types

# Tensor axis of each dim in the (z, x, y) storage order.
AXIS = {0: 1, 1: 2, 2: 0}


class BlockLayout:
  """Block coordinates and neighbours of the replicas array."""

  def __init__(self, replicas: np.ndarray, periodic: Sequence[bool]):
    self.replicas = np.asarray(replicas)
    if self.replicas.ndim != 3:
      raise ValueError('replicas must be a 3-D array (cx, cy, cz).')
    self.shape = self.replicas.shape
    self.periodic = [bool(p) for p in periodic]

  @property
  def n_blocks(self) -> int:
    return int(self.replicas.size)

  def coords(self, rid: int):
    where = np.argwhere(self.replicas == rid)
    if len(where) != 1:
      raise ValueError(f'Replica id {rid} is not in the replicas array.')
    return tuple(int(c) for c in where[0])

  def neighbour(self, rid: int, dim: int, side: int) -> Optional[int]:
    """Block across `side` (0 low, 1 high) of `dim`, or None where the side
    takes a boundary condition (or the dim is not split)."""
    n = self.shape[dim]
    if n == 1:
      return None
    c = list(self.coords(rid))
    c[dim] += -1 if side == 0 else 1
    if c[dim] < 0 or c[dim] >= n:
      if not self.periodic[dim]:
        return None
      c[dim] %= n
    return int(self.replicas[tuple(c)])


def slab(t: torch.Tensor, dim: int, hw: int, which: str, side: int):
  """View of `hw` layers along `dim`: which='interior' gives the interior
  layers next to `side`, which='halo' the halo layers of `side`."""
  ax = AXIS[dim]
  n = t.shape[ax] - 2 * hw
  if which == 'interior':
    lo = hw if side == 0 else n
  else:
    lo = 0 if side == 0 else n + hw
  return t.narrow(ax, lo, hw)


def _rescale_primitive(fields, via, dim, hw, side):
  """Halo of a field whose BC is given on its primitive: the reference
  exchanges phi/rho and multiplies back by rho (boundary.py:516-531), so the
  halo holds rho*(f/rho), with 0 where rho is 0."""
  rho = slab(fields[0], dim, hw, 'halo', side)
  for f, v in zip(fields, via):
    if v:
      h = slab(f, dim, hw, 'halo', side)
      q = torch.where(rho == 0, torch.zeros_like(h), h / rho)
      h.copy_(rho * q)


class _Exchange:
  """Shared driver: for each dim, boundary conditions on the block's own
  sides, then the transfer between blocks on the inner sides."""

  def __init__(self, layout: BlockLayout, hw: int,
               bc_fill: Callable[[int, List[torch.Tensor], int], None],
               via_primitive: Sequence[int] = (0, 0, 0, 0, 0)):
    self.layout = layout
    self.hw = hw
    self.bc_fill = bc_fill
    self.via = list(via_primitive)

  def _transfer(self, blocks, rids, dim):
    raise NotImplementedError

  def fill(self, blocks: List[List[torch.Tensor]], rids: Sequence[int]):
    """Complete halo update of the fields of every block held here."""
    for dim in range(3):
      for b, rid in zip(blocks, rids):
        self.bc_fill(rid, b, dim)
      self._transfer(blocks, rids, dim)

  def min_all(self, t: torch.Tensor) -> None:
    raise NotImplementedError


class LocalExchange(_Exchange):
  """Every block in this process: inner sides are copied between blocks."""

  def _transfer(self, blocks, rids, dim):
    index = {rid: i for i, rid in enumerate(rids)}
    for b, rid in zip(blocks, rids):
      for side in (0, 1):
        nb = self.layout.neighbour(rid, dim, side)
        if nb is None:
          continue
        src = blocks[index[nb]]
        for f, g in zip(b, src):
          slab(f, dim, self.hw, 'halo', side).copy_(
              slab(g, dim, self.hw, 'interior', 1 - side))
        if any(self.via):
          _rescale_primitive(b, self.via, dim, self.hw, side)

  def min_all(self, ts: Sequence[torch.Tensor]) -> None:
    m = torch.stack([t.reshape(()) for t in ts]).min()
    for t in ts:
      t.fill_(m)


class DistExchange(_Exchange):
  """One block per process over torch.distributed (default group).

  Messages between two blocks in one direction are matched in issue order
  (NCCL has no tags), so every process issues, per dim: send low slab, receive
  high halo, send high slab, receive low halo."""

  def _transfer(self, blocks, rids, dim):
    import torch.distributed as dist
    (b,), (rid,) = blocks, rids
    nbs = [self.layout.neighbour(rid, dim, s) for s in (0, 1)]
    if nbs == [None, None]:
      return
    hw = self.hw
    ops, recvs = [], []
    for send_side, recv_side in ((0, 1), (1, 0)):
      if nbs[send_side] is not None:
        buf = torch.stack([slab(f, dim, hw, 'interior', send_side).contiguous()
                           for f in b])
        ops.append(dist.P2POp(dist.isend, buf, nbs[send_side],
                              tag=2 * dim + send_side))
      if nbs[recv_side] is not None:
        shape = (len(b),) + tuple(slab(b[0], dim, hw, 'halo', recv_side).shape)
        rbuf = torch.empty(shape, dtype=b[0].dtype, device=b[0].device)
        ops.append(dist.P2POp(dist.irecv, rbuf, nbs[recv_side],
                              tag=2 * dim + (1 - recv_side)))
        recvs.append((recv_side, rbuf))
    for req in dist.batch_isend_irecv(ops):
      req.wait()
    for side, rbuf in recvs:
      for f, r in zip(b, rbuf):
        slab(f, dim, hw, 'halo', side).copy_(r)
      if any(self.via):
        _rescale_primitive(b, self.via, dim, hw, side)

  def min_all(self, ts: Sequence[torch.Tensor]) -> None:
    import torch.distributed as dist
    (t,) = ts
    dist.all_reduce(t, op=dist.ReduceOp.MIN)


def periodic_dims(cfg) -> List[bool]:
  """Per dim, whether the conserved fields' BCs are periodic there; every
  field must agree (one transfer serves all five)."""
  bc = cfg.bc.get('cell_averages', {})
  out = []
  for d in types.DIMS:
    kinds = set()
    for name in types.BASE_CONSERVATIVE:
      spec = bc.get(name, bc.get(types.conservative_to_primitive_name(name)))
      if spec is None or d not in spec:
        kinds.add(False)
        continue
      kinds.add(any(getattr(v[0], 'value', v[0]) == 0
                    for v in spec[d].values()))
    if len(kinds) != 1:
      raise NotImplementedError(
          f'Fields disagree on whether dim {d} is periodic; a decomposed '
          'grid needs one periodicity per dim.')
    out.append(kinds.pop())
  return out


def localize_bc(bc: Dict, replicas: np.ndarray, rid: int, hw: int,
                global_interior: Sequence[int]) -> Dict:
  """The BC dict of block `rid`: per-layer Dirichlet planes given for the
  whole grid (with halos) are cut to the block's window; planes already of
  the block's size and scalar values pass through."""
  nz, nx, ny = global_interior
  c = np.argwhere(np.asarray(replicas) == rid)[0]
  cx, cy, cz = np.asarray(replicas).shape
  lz, lx, ly = nz // cz, nx // cx, ny // cy
  win = {'z': (int(c[2]) * lz, lz + 2 * hw), 'x': (int(c[0]) * lx, lx + 2 * hw),
         'y': (int(c[1]) * ly, ly + 2 * hw)}
  full = {'z': nz + 2 * hw, 'x': nx + 2 * hw, 'y': ny + 2 * hw}
  axes = {'x': ('z', 'y'), 'y': ('z', 'x'), 'z': ('x', 'y')}

  def cut(v, dim):
    if isinstance(v, torch.Tensor):
      v = v.detach().cpu().numpy()
    a = np.asarray(v)
    ea, eb = axes[dim]
    if a.ndim == 2 and a.shape == (full[ea], full[eb]):
      (oa, na), (ob, nb) = win[ea], win[eb]
      return np.ascontiguousarray(a[oa:oa + na, ob:ob + nb])
    return v

  out = {}
  for name, spec in bc.items():
    if not isinstance(spec, dict):
      out[name] = spec
      continue
    nspec = {}
    for dim, sides in spec.items():
      nsides = {}
      for side, val in (sides or {}).items():
        if len(val) > 1 and not np.isscalar(val[1]):
          layers = val[1]
          if isinstance(layers, (list, tuple)):
            nsides[side] = (val[0], [cut(v, dim) for v in layers]) + tuple(val[2:])
          else:
            nsides[side] = (val[0], cut(layers, dim)) + tuple(val[2:])
        else:
          nsides[side] = val
      nspec[dim] = nsides
    out[name] = nspec
  return out


def masked_bcs(solver, layout: BlockLayout, rid: int, nat):
  """Per dim, the solver's BC table restricted to that dim's sides that take
  a boundary condition (inner sides and other dims set to NONE)."""
  out = []
  for dim in range(3):
    arr = (nat.SwcFieldBC * len(solver.bcs))()
    ctypes.memmove(arr, solver.bcs, ctypes.sizeof(arr))
    for fi in range(len(solver.bcs)):
      for d in range(3):
        for s in range(2):
          inner = d == dim and layout.neighbour(rid, d, s) is not None
          if d != dim or inner:
            arr[fi].side[d][s].kind = nat.SWC_BC_NONE
    out.append(arr)
  return out
