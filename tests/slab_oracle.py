"""The oracle on z-slabs of a full-size grid, in parallel host processes.

A one-step comparison at the benchmark sizes (256^3, 512x512x256) does not
fit the NumPy oracle in one process, so each slab of interior z planes
[z0, z1) is stepped on its own, cut out of the full state with PAD extra
planes on each side: one SSP-RK3 step reads 3 cells per stage along z, so
planes more than 9 away from a cut are exactly what the whole-grid step
gives (the cut's halo is left as it is, BC kind NONE). Sides on the grid's
own z walls keep the grid's BC and its halo planes. Potential energy and
helper states are sliced from the whole grid's.

Test infrastructure: only tests import this module. The pool uses `spawn`.
"""

import copy
import multiprocessing as mp
import os
from typing import Dict, List, Sequence, Tuple

import numpy as np

from oracle import swirlc_oracle as orc

PAD = 9  # 3 stages x stencil radius 3


def _worker(payload):
  ocfg, cons, pe, helper, dt, lo, hi, hw = payload
  out = orc.rk3(cons, dt, lambda s: orc.rhs(s, ocfg, helper, pe=pe))
  return {k: np.ascontiguousarray(v[lo:hi, hw:-hw, hw:-hw])
          for k, v in out.items()}


def _slab_cfg(ocfg, z_lo_wall: bool, z_hi_wall: bool):
  c = copy.deepcopy(ocfg)
  for dims in c.bc['cell_averages'].values():
    z = dims.get('z')
    lo = z[0] if (z and z_lo_wall and orc.bc_kind(z[0][0]) != orc.PERIODIC) \
        else (orc.NONE,)
    hi = z[1] if (z and z_hi_wall and orc.bc_kind(z[1][0]) != orc.PERIODIC) \
        else (orc.NONE,)
    dims['z'] = {0: lo, 1: hi}
  return c


def one_step(ocfg, state: Dict[str, np.ndarray], dt: float,
             slabs: Sequence[Tuple[int, int]], dtype=np.float32,
             helper: Dict[str, np.ndarray] = None,
             procs: int = 0) -> List[Dict[str, np.ndarray]]:
  """Per slab (z0, z1): the oracle's state after one RK3 step of size dt on
  interior planes [z0, z1), interior x and y only."""
  hw = ocfg.halo_width
  nz = state['rho'].shape[0] - 2 * hw
  periodic_z = all(
      orc.bc_kind(d['z'][0][0]) == orc.PERIODIC
      for d in ocfg.bc['cell_averages'].values() if 'z' in d)
  st = {k: v.astype(dtype) for k, v in state.items()}
  pe_full = orc.potential_energy(ocfg, st['rho'].shape, dtype)
  tasks = []
  for z0, z1 in slabs:
    if periodic_z:
      idx = (np.arange(z0 - PAD - hw, z1 + PAD + hw) % nz) + hw
      lo_wall = hi_wall = False
    else:
      a = max(0, z0 - PAD)
      b = min(nz + 2 * hw, z1 + PAD + 2 * hw)
      idx = np.arange(a, b)
      lo_wall, hi_wall = a == 0, b == nz + 2 * hw
    cons = {k: np.ascontiguousarray(v[idx]) for k, v in st.items()}
    pe = np.ascontiguousarray(pe_full[idx])
    hp = ({k: np.ascontiguousarray(v.astype(dtype)[idx])
           for k, v in helper.items()} if helper else None)
    lo = int(np.nonzero(idx == z0 + hw)[0][0])
    tasks.append((_slab_cfg(ocfg, lo_wall, hi_wall), cons, pe, hp,
                  dtype(dt), lo, lo + (z1 - z0), hw))
  if not procs:
    try:
      procs = len(os.sched_getaffinity(0))
    except AttributeError:
      procs = os.cpu_count() or 1
  procs = max(1, min(procs, len(tasks)))
  if procs == 1:
    return [_worker(t) for t in tasks]
  with mp.get_context('spawn').Pool(procs) as pool:
    return pool.map(_worker, tasks)
