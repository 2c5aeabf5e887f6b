"""Gradients of whole runs: the discrete adjoint of the fused RK stages.

The reference differentiates its TensorFlow graph with GradientTape. Here a
run of SSP-RK3 (rk3.py:87-120) or RK2 (rk2.py:69-86) steps is reversed with
the stage vector-Jacobian product of the library (`swc_rk_stage_vjp`), with
checkpointing: the forward run keeps the state every `checkpoint_every`
steps; the backward sweep recomputes one segment at a time, keeping that
segment's stage states, and walks back through it. The time steps are those
of the forward run and are held fixed (not differentiated), as in the
reference's KH set-up where dt is computed once on the host.

For a step u -> u' with stages
  u1 = u + dt L(u),  u2 = 3/4 u + 1/4 (u1 + dt L(u1)),
  u' = 1/3 u + 2/3 (u2 + dt L(u2)),
the reverse of a cotangent g of u' is
  g2 = 2/3 g + V(u2, g, 2/3 dt),   g1 = 1/4 g2 + V(u1, g2, 1/4 dt),
  g_u = 1/3 g + 3/4 g2 + g1 + V(u, g1, dt),
where V(uk, lam, beta) = beta H^T J_L(H uk)^T lam (the library call). The
derivative with respect to the kinematic viscosity nu is accumulated by the
same calls.
"""

import ctypes
from typing import List, Optional, Sequence, Tuple

import torch

from swirlc_b200 import _native as nat
from swirlc_b200 import engine


class RunAdjoint:
  """A forward run with checkpoints and its reverse sweep for one solver.

  Args:
    solver: an `engine.Solver` (WENO5 or MUSCL, HLL or HLLC, optionally
      viscous; no transported scalars).
    checkpoint_every: steps between stored states; 0 keeps every step's
      stage states during the forward run instead (no recomputation in the
      backward sweep; memory: steps x 3 states of the fields).
    scheme: 'rk3' or 'rk2'.
    steps: when known, the run length, so that the stage buffers (reused by
      every run and sweep) are allocated here rather than during the run.
  """

  def __init__(self, solver: engine.Solver, checkpoint_every: int = 20,
               scheme: str = 'rk3', steps: int = 0):
    if scheme not in ('rk3', 'rk2'):
      raise NotImplementedError(f'"{scheme}" is not implemented as an '
                                '"time_integration_scheme".')
    if checkpoint_every < 0:
      raise ValueError('checkpoint_every must be >= 0.')
    self.s = solver
    self.k = int(checkpoint_every)
    self.order = 3 if scheme == 'rk3' else 2
    self.checkpoints: List[List[torch.Tensor]] = []
    self.dts: List[float] = []
    # Incremented by every run(): the checkpoints, dts and stage buffers of
    # a runner belong to its latest run only.
    self.generation = 0
    self._scratch = [torch.empty(solver.shape, dtype=solver.dtype,
                                 device=solver.device)
                     for _ in range(nat.SWC_VJP_SCRATCH)]
    self._g = [solver.new_fields(zero=True) for _ in range(4)]
    self._nu_bar = torch.zeros(1, dtype=torch.float64, device=solver.device)
    self._pool: List = []  # per-step stage buffers, reused
    self._tmp = None       # stage buffers of steps that keep nothing
    self._u = None         # working state of the recomputed segment
    self._ckpt_pool: List = []  # checkpoint states, reused
    # Index of the segment whose stage states the last run() left in
    # self._pool (the final one), or -1: its reverse needs no recompute.
    self._kept = -1
    if steps:
      self._reserve(steps if self.k == 0 else min(self.k, steps))
      if self.k:
        self._reserve_checkpoints((steps + self.k - 1) // self.k)
      if self.k and steps > self.k:
        # Stage buffers of the steps that keep nothing, and the working state
        # of the segment recompute: allocated here, not inside a run.
        self._tmp = self._new_buffers()
        self._u = solver.new_fields(zero=False)

  # ------------------------------------------------------------- forward
  def _new_buffers(self):
    n = 3 if self.order == 3 else 2
    return tuple(self.s.new_fields(zero=False) for _ in range(n))

  def _reserve(self, n: int) -> None:
    while len(self._pool) < n:
      self._pool.append(self._new_buffers())

  def _reserve_checkpoints(self, n: int) -> None:
    while len(self._ckpt_pool) < n:
      self._ckpt_pool.append(self.s.new_fields(zero=False))

  def _step(self, u, i, buf=None):
    """Step i in place on u with its fixed dt; the halo-filled stage states
    (u, u1, u2) are left in `buf` (scratch buffers when None)."""
    s = self.s
    if buf is None:
      if self._tmp is None:
        self._tmp = self._new_buffers()
      buf = self._tmp
    dtt = self._dt_dev[i:i + 1]
    s.fill_halos(u)
    u0, w1 = buf[0], buf[1]
    for a, b in zip(u0, u):
      a.copy_(b)
    s.stage(u0, None, w1, nat.SWC_OUT_EULER, dt=dtt)
    s.fill_halos(w1)
    if self.order == 3:
      w2 = buf[2]
      s.stage(w1, u0, w2, nat.SWC_OUT_CONVEX, 0.75, 0.25, dt=dtt)
      s.fill_halos(w2)
      s.stage(w2, u0, u, nat.SWC_OUT_CONVEX, 1.0 / 3.0, 2.0 / 3.0, dt=dtt)
    else:
      s.stage(w1, u0, u, nat.SWC_OUT_AVERAGE, 0.5, 0.0, dt=dtt)
    return buf

  def run(self, fields: Sequence[torch.Tensor],
          dts: Sequence[float]) -> List[torch.Tensor]:
    """Advances a copy of `fields` by len(dts) steps, keeping checkpoints."""
    self.s.check_fields(fields)
    self.generation += 1
    self.dts = [float(d) for d in dts]
    # Every step's dt on the device in one copy: a copy per step from
    # pageable host memory would wait for the stream each time.
    self._dt_dev = torch.tensor(self.dts or [0.0], dtype=torch.float64,
                                device=self.s.device)
    u = [f.detach().clone() for f in fields]
    self.checkpoints = []
    self._kept = -1
    if self.k == 0:
      self._reserve(len(self.dts))
    else:
      self._reserve(min(self.k, len(self.dts)))
    # The final segment's stage states stay in the pool: the reverse sweep
    # starts there, so it needs no recompute of that segment.
    last_seg = (len(self.dts) - 1) // self.k if self.k and self.dts else -1
    for i in range(len(self.dts)):
      if self.k == 0:
        self._step(u, i, self._pool[i])
        continue
      if i % self.k == 0:
        c = i // self.k
        self._reserve_checkpoints(c + 1)
        for a, b in zip(self._ckpt_pool[c], u):
          a.copy_(b)
        self.checkpoints.append(self._ckpt_pool[c])
      if i // self.k == last_seg:
        self._step(u, i, self._pool[i - last_seg * self.k])
      else:
        self._step(u, i)
    self._kept = last_seg
    if self.k == 0:
      self.checkpoints = [None]
    self.s.fill_halos(u)
    return u

  # ------------------------------------------------------------ backward
  def _vjp(self, uk, lam, alpha, beta, out, x1=None, c1=0.0, x2=None,
           c2=0.0) -> None:
    """out = alpha*lam + c1*x1 + c2*x2 + beta*H^T J^T lam (interior)."""
    s = self.s
    nat.check(nat.load().swc_rk_stage_vjp(
        ctypes.byref(s.grid), ctypes.byref(s.scheme), s.bcs,
        nat.ptr_array(uk), nat.ptr_array(lam), float(alpha), float(beta),
        nat.ptr_array(x1) if x1 is not None else None, float(c1),
        nat.ptr_array(x2) if x2 is not None else None, float(c2),
        nat.ptr_array(out), self._nu_bar.data_ptr(),
        nat.ptr_array(self._scratch), nat.stream_ptr()), 'stage vjp')

  def _reverse_step(self, stages, dt, g, gn, g2, g1) -> None:
    """gn = cotangent of the step's input for the cotangent g of its
    output: one swc_rk_step_vjp call (its two or three stage adjoints are
    the `_vjp` calls of `_reverse_step_by_stage`)."""
    s = self.s
    flat = [f for st in stages[:self.order] for f in st]
    nat.check(nat.load().swc_rk_step_vjp(
        ctypes.byref(s.grid), ctypes.byref(s.scheme), s.bcs, self.order,
        nat.ptr_array(flat), float(dt), nat.ptr_array(g), nat.ptr_array(gn),
        nat.ptr_array(list(g1) + list(g2)), self._nu_bar.data_ptr(),
        nat.ptr_array(self._scratch), nat.stream_ptr()), 'step vjp')

  def _reverse_step_by_stage(self, stages, dt, g, gn, g2, g1) -> None:
    """The same reverse step as three (RK2: two) stage adjoints."""
    if self.order == 3:
      u0, u1, u2 = stages
      self._vjp(u2, g, 2.0 / 3.0, 2.0 / 3.0 * dt, g2)
      self._vjp(u1, g2, 0.25, 0.25 * dt, g1)
      self._vjp(u0, g1, 1.0, dt, gn, g, 1.0 / 3.0, g2, 0.75)
    else:
      u0, u1 = stages
      self._vjp(u1, g, 0.5, 0.5 * dt, g1)
      self._vjp(u0, g1, 1.0, dt, gn, g, 0.5)

  def backward(self, grad_out: Sequence[torch.Tensor]
               ) -> Tuple[List[torch.Tensor], float]:
    """Cotangent of the initial fields and d/dnu for a cotangent of the final
    fields (interior cells; halos are ignored)."""
    if not self.checkpoints:
      raise RuntimeError('backward() needs a run() first.')
    hw = self.s.hw
    inner = (slice(hw, -hw),) * 3
    g, gn, g2, g1 = self._g
    for dst, src in zip(g, grad_out):
      dst.zero_()
      dst[inner] = src[inner].to(self.s.dtype)
    self._nu_bar.zero_()
    nsteps = len(self.dts)
    if self.k == 0:
      for i in reversed(range(nsteps)):
        self._reverse_step(self._pool[i], self.dts[i], g, gn, g2, g1)
        g, gn = gn, g
    else:
      self._reserve(min(self.k, nsteps))
      for c in reversed(range(len(self.checkpoints))):
        first = c * self.k
        last = min(first + self.k, nsteps)
        if c != self._kept:
          if self._u is None:
            self._u = self.s.new_fields(zero=False)
          u = self._u
          for a, b in zip(u, self.checkpoints[c]):
            a.copy_(b)
          for i in range(first, last):
            self._step(u, i, self._pool[i - first])
        # The pool now holds segment c; later sweeps recompute everything.
        self._kept = -1
        for i in reversed(range(first, last)):
          self._reverse_step(self._pool[i - first], self.dts[i], g, gn, g2,
                             g1)
          g, gn = gn, g
    return [x.clone() for x in g], float(self._nu_bar.item())


class _Run(torch.autograd.Function):
  """Forward run / reverse sweep as one autograd node.

  A runner holds the checkpoints of its latest run only, so it serves one
  outstanding simulate() at a time: backward raises if the runner has run
  again since this node's forward (use one RunAdjoint per live graph).
  """

  @staticmethod
  def forward(ctx, runner, dts, nu, *fields):
    runner.s.scheme.nu = float(nu)
    out = runner.run(fields, dts)
    ctx.runner = runner
    ctx.generation = runner.generation
    ctx.nu_value = float(nu)
    ctx.nu_meta = (nu.dtype, nu.device)
    return tuple(out)

  @staticmethod
  def backward(ctx, *grads):
    runner = ctx.runner
    if runner.generation != ctx.generation:
      raise RuntimeError(
          'RunAdjoint has run again since this simulate() call; its '
          'checkpoints now belong to the later run. Use one RunAdjoint per '
          'simulate() whose backward is still pending.')
    runner.s.scheme.nu = ctx.nu_value
    grads = [torch.zeros_like(runner._g[0][0]) if g is None else g
             for g in grads]
    gin, nub = runner.backward(grads)
    dtype, device = ctx.nu_meta
    return (None, None, torch.tensor(nub, dtype=dtype, device=device),
            *gin)


def simulate(runner: RunAdjoint, fields: Sequence[torch.Tensor],
             dts: Sequence[float], nu: torch.Tensor) -> Tuple[torch.Tensor, ...]:
  """Differentiable run: the final fields as a function of the initial
  fields and of the kinematic viscosity `nu` (a 0-d tensor)."""
  return _Run.apply(runner, list(dts), nu, *fields)


def vorticity_energy(fields: Sequence[torch.Tensor], hw: int, dx: float,
                     dy: float, dz: float) -> torch.Tensor:
  """Loss of the adjoint benchmark: integral of |omega|^2 / 2 over the
  periodic interior, omega = curl(u) by central differences, u = rho_u/rho.
  Axes of the stored fields are (z, x, y)."""
  sl = (slice(hw, -hw),) * 3
  rho, ru, rv, rw = (f[sl] for f in fields[:4])
  u, v, w = ru / rho, rv / rho, rw / rho

  def d(f, axis, h):
    return (torch.roll(f, -1, axis) - torch.roll(f, 1, axis)) / (2.0 * h)

  wx = d(w, 2, dy) - d(v, 0, dz)
  wy = d(u, 0, dz) - d(w, 1, dx)
  wz = d(v, 1, dx) - d(u, 2, dy)
  return 0.5 * (wx * wx + wy * wy + wz * wz).sum() * (dx * dy * dz)
