"""Batched time stepping of many independent grids ("members").

The reference advances one grid per program (`Simulation.step`,
simulation.py:68-105); a parameter sweep or an ensemble of small problems
then pays the full launch sequence of a step once per member. Here every
member is configured exactly as for `Simulation` (a config dict or
`SwirlCParameters` plus its state dict) and `swc_batch_step` advances all of
them by one step with one batched halo pass per dim and one batched stage
launch per tile shape per RK stage. Each member keeps its own device clock,
so each takes its own CFL time step.

All members must share the numerical scheme (interpolation, limiter, Riemann
solver, diffusion and transport constants, gravity vector); grids, boundary
conditions and initial states are free.
"""

import ctypes
from typing import Dict, List, Optional, Sequence, Tuple

import torch

from swirlc_b200 import _native as nat
from swirlc_b200 import engine
from swirlc_b200.common import types
from swirlc_b200.core import parameter
from swirlc_b200.physics import physics_models as pm_lib

# SwcBatchMember.tile codes. TILE_AUTO (16x16) reproduces the single-grid
# step bit for bit; TILE_8X32 suits members at most 8 cells wide in y and can
# differ from it in the last bit.
TILE_AUTO, TILE_16X16, TILE_8X32 = 0, 1, 2

_SHARED = ('dtype', 'interp', 'limiter', 'riemann', 'diffusion', 'nscalars',
           'gravity_mask', 'nu', 'pr')


class BatchStepper:
  """In-place time loop over a batch of members with per-member clocks.

  Args:
    members: sequence of (config, state); config is a user config dict or a
      `SwirlCParameters`, state maps the conserved names to arrays/tensors of
      shape (nz + 2h, nx + 2h, ny + 2h).
    dtype: torch.float32 or torch.float64.
    scheme: 'rk3' or 'rk2' (shared by all members).
    dt, cfl, t_end: per-member step control as in `engine.Stepper`; when
      None, each member's config value is used (`dt`, `cfl`, `t_end`).
  """

  def __init__(self, members: Sequence[Tuple[object, Dict]],
               dtype: torch.dtype = torch.float32, scheme: str = 'rk3',
               dt: Optional[float] = None, cfl: Optional[float] = None,
               t_end: Optional[float] = None):
    if not members:
      raise ValueError('A batch needs at least one member.')
    if scheme not in ('rk3', 'rk2'):
      raise NotImplementedError(f'"{scheme}" is not implemented as an '
                                '"time_integration_scheme".')
    self.order = 3 if scheme == 'rk3' else 2
    self.dtype = dtype
    self.solvers: List[engine.Solver] = []
    self.u: List[List[torch.Tensor]] = []
    self.work: List[List[torch.Tensor]] = []
    self.clocks: List[torch.Tensor] = []
    for i, (cfg, state) in enumerate(members):
      if not isinstance(cfg, parameter.SwirlCParameters):
        cfg = parameter.SwirlCParameters(cfg)
      pm = pm_lib.PhysicsModels(cfg)
      fields = [torch.as_tensor(state[k]).to(device='cuda', dtype=dtype)
                .contiguous() for k in types.BASE_CONSERVATIVE]
      solver = engine.Solver(cfg, pm, fields[0].shape, dtype)
      solver.check_fields(fields)
      if self.solvers:
        ref = self.solvers[0].scheme
        for name in _SHARED:
          if getattr(solver.scheme, name) != getattr(ref, name):
            raise ValueError(
                f'Member {i} differs from member 0 in "{name}"; all members '
                'of a batch share the numerical scheme.')
        if list(solver.scheme.g) != list(ref.g):
          raise ValueError(f'Member {i} has another gravity vector.')
      self.solvers.append(solver)
      self.u.append(fields)
      self.work.append(solver.new_fields(zero=False) +
                       solver.new_fields(zero=False))
      clock = torch.zeros(6, dtype=torch.float64, device=solver.device)
      mdt = float(cfg.dt if dt is None else dt)
      mcfl = float((getattr(cfg, 'cfl', 0.0) or 0.0) if cfl is None else cfl)
      mend = float((getattr(cfg, 't_end', 0.0) or 0.0) if t_end is None
                   else t_end)
      clock[1] = mdt
      clock[2] = 1e300
      clock[3] = mcfl
      clock[4] = mend
      if mcfl > 0.0:
        solver.cfl_reduce(fields, clock[2:3])
      self.clocks.append(clock)
    self.scheme = nat.SwcScheme.from_buffer_copy(self.solvers[0].scheme)
    for d in range(3):
      self.scheme.pe_axis[d] = None
    self.table = (nat.SwcBatchMember * len(self.solvers))()
    for i, s in enumerate(self.solvers):
      m = self.table[i]
      m.grid = nat.SwcGrid.from_buffer_copy(s.grid)
      for v in range(5):
        m.u[v] = self.u[i][v].data_ptr()
      for v in range(10):
        m.work[v] = self.work[i][v].data_ptr()
      for d in range(3):
        m.pe_axis[d] = s.scheme.pe_axis[d]
      for v in range(5):
        m.bcs[v] = nat.SwcFieldBC.from_buffer_copy(s.bcs[v])
      m.clock = self.clocks[i].data_ptr()
      m.tile = TILE_AUTO
      m.zseg = 0
    self.graph: Optional[torch.cuda.CUDAGraph] = None
    self.graph_steps = 0

  # ------------------------------------------------------------- stepping
  @property
  def n_members(self) -> int:
    return len(self.solvers)

  def cells(self) -> int:
    """Interior cells over all members."""
    return sum(s.nx * s.ny * s.nz for s in self.solvers)

  def set_launch(self, tiles: Optional[Sequence[int]] = None,
                 zsegs: Optional[Sequence[int]] = None) -> None:
    """Per-member tile codes (TILE_*) and z planes per CTA (0 = auto)."""
    if self.graph is not None:
      raise RuntimeError('set_launch after capture(); capture again.')
    for i in range(self.n_members):
      if tiles is not None:
        self.table[i].tile = int(tiles[i])
      if zsegs is not None:
        self.table[i].zseg = int(zsegs[i])

  def _launch_step(self) -> None:
    nat.check(nat.load().swc_batch_step(
        ctypes.byref(self.scheme), self.order, self.n_members, self.table,
        nat.stream_ptr()), 'batch step')

  def capture(self, steps: int = 1) -> None:
    """Captures `steps` batch steps in one CUDA graph (run eagerly once
    first, so that every kernel variant is loaded)."""
    self.graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
      with torch.cuda.graph(self.graph, stream=side):
        for _ in range(steps):
          self._launch_step()
    torch.cuda.current_stream().wait_stream(side)
    self.graph_steps = steps

  def step(self, n: int = 1, check: bool = False) -> None:
    """Advances every member by n steps (graph replays when captured; n must
    then be a multiple of the captured step count). With `check`, waits and
    raises FloatingPointError naming the first member whose new state holds
    a non-finite rho, p or rho_e (swc_clock_status on its clock)."""
    if self.graph is None:
      for _ in range(n):
        self._launch_step()
    else:
      if n % self.graph_steps:
        raise ValueError(f'{n} steps is not a multiple of the captured '
                         f'{self.graph_steps}.')
      for _ in range(n // self.graph_steps):
        self.graph.replay()
    if check:
      lib = nat.load()
      for i, c in enumerate(self.clocks):
        nat.check(lib.swc_clock_status(c.data_ptr(), nat.stream_ptr()),
                  f'batch member {i}')

  # ------------------------------------------------------------ autotuner
  def _snapshot(self):
    return ([[f.clone() for f in u] for u in self.u],
            [c.clone() for c in self.clocks])

  def _restore(self, snap) -> None:
    us, cs = snap
    for u, su in zip(self.u, us):
      for f, sf in zip(u, su):
        f.copy_(sf)
    for c, sc in zip(self.clocks, cs):
      c.copy_(sc)

  def autotune(self, candidates: Optional[Sequence[Tuple[int, int]]] = None,
               steps: int = 2, reps: int = 3) -> Dict:
    """Times launch policies on this batch and keeps the fastest.

    A policy is (small_ny, zseg): members with ny <= small_ny get the 8x32
    tile, the others 16x16; zseg is the z planes per CTA (0 = the library's
    choice). Each candidate runs `steps` eager steps `reps` times from the
    same saved state; the state and clocks are restored afterwards.
    """
    if self.graph is not None:
      raise RuntimeError('autotune before capture().')
    if candidates is None:
      narrow = 8 if self.dtype == torch.float32 or self.scheme.interp != 0 \
          else 0
      candidates = [(sm, z) for sm in sorted({0, narrow})
                    for z in (0, 8, 16, 32)]
    snap = self._snapshot()
    start, stop = (torch.cuda.Event(enable_timing=True) for _ in range(2))
    results = []
    for small, zseg in candidates:
      tiles = [TILE_8X32 if s.ny <= small else TILE_16X16
               for s in self.solvers]
      self.set_launch(tiles, [zseg] * self.n_members)
      self._launch_step()  # load variants
      best = float('inf')
      for _ in range(reps):
        self._restore(snap)
        torch.cuda.synchronize()
        start.record()
        for _ in range(steps):
          self._launch_step()
        stop.record()
        torch.cuda.synchronize()
        best = min(best, start.elapsed_time(stop) / steps)
      results.append(((small, zseg), best))
    self._restore(snap)
    (small, zseg), ms = min(results, key=lambda r: r[1])
    tiles = [TILE_8X32 if s.ny <= small else TILE_16X16 for s in self.solvers]
    self.set_launch(tiles, [zseg] * self.n_members)
    torch.cuda.synchronize()
    return {'small_ny': small, 'zseg': zseg, 'ms_per_step': ms,
            'results': results}

  # ---------------------------------------------------------------- state
  def time(self, i: int) -> float:
    return float(self.clocks[i][0].item())

  def steps_done(self, i: int) -> int:
    return int(self.clocks[i][5:6].view(torch.int64).item())

  def state(self, i: int) -> Dict[str, torch.Tensor]:
    return dict(zip(types.BASE_CONSERVATIVE, self.u[i]))


def sequential_plain(members: Sequence[Tuple[object, Dict]], steps: int,
                     dtype: torch.dtype = torch.float32) -> Dict:
  """Reference point for the batch: the same members advanced one after
  another, each by its own `engine.Stepper` replaying a one-step CUDA graph.
  Returns the summed device time and cell-updates/s."""
  total_ms = 0.0
  cells = 0
  start, stop = (torch.cuda.Event(enable_timing=True) for _ in range(2))
  for cfg, state in members:
    if not isinstance(cfg, parameter.SwirlCParameters):
      cfg = parameter.SwirlCParameters(cfg)
    pm = pm_lib.PhysicsModels(cfg)
    fields = [torch.as_tensor(state[k]).to(device='cuda', dtype=dtype)
              .contiguous() for k in types.BASE_CONSERVATIVE]
    solver = engine.Solver(cfg, pm, fields[0].shape, dtype)
    cfl = float(getattr(cfg, 'cfl', 0.0) or 0.0)
    st = engine.Stepper(solver, fields, dt=float(cfg.dt), cfl=cfl)
    st.step(1)
    st.capture()
    torch.cuda.synchronize()
    start.record()
    st.step(steps)
    stop.record()
    torch.cuda.synchronize()
    total_ms += start.elapsed_time(stop)
    cells += solver.nx * solver.ny * solver.nz
    del st, solver, fields
  return {'ms': total_ms, 'cell_updates_per_s': cells * steps / (total_ms * 1e-3)}

