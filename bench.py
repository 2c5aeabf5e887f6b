"""Benchmark: SSP-RK3 cell-updates/s of the 3-D Kelvin-Helmholtz set-up.

Workload (one "step" = one SSP-RK3 step = 3 fused stage passes): periodic
unit cube of 256^3 interior cells, float32, WENO5-JS + HLLC + viscous
(nu = 1e-4, Pr = 0.7), CFL 0.5 with the time step reduced on the device.
Seeded synthetic initial condition (swirlc_b200.configs.kelvin_helmholtz).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload kh256|riemann_batch|adjoint|sod|bubble]

Under torchrun each rank advances its own 256^3 domain (weak scaling,
replicas; the halo exchange of a decomposed domain is a separate path).
`value` is the whole-job cell-updates/s (all ranks' cells x K / max time).
`e2e` times the public API call `Simulation.step` with the state copied from
pinned host memory and the result copied back every step.
`--impl reference` times the CPU oracle (the NumPy restatement of the
reference path) on this host's cores over a bounded sample of the same
workload; the reference's own TensorFlow path cannot run here.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

N_CELLS_EDGE = 256
ALG_BYTES_PER_CELL_UPDATE = 160  # fp32: 40 + 60 + 60 B over the 3 stages
METRIC = 'RK3 cell-updates/s at 256^3 fp32 (% HBM roofline)'
UNIT = 'cell-updates/s'


def _env_rank():
  return (int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1')),
          int(os.environ.get('LOCAL_RANK', '0')))


def _peaks():
  path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
  try:
    with open(path) as f:
      p = json.load(f)
    return float(p['hbm_gbs']), 'measured'
  except (OSError, KeyError, ValueError):
    return 6650.0, 'fallback'


def _profile_figure(key):
  """A per-cell figure of the stage kernel from the committed ncu summary."""
  path = os.path.join(ROOT, 'profiles', 'stage_kernel_kh256.txt')
  try:
    with open(path) as f:
      for line in f:
        if line.startswith(key + ':'):
          return float(line.split(':', 1)[1])
  except OSError:
    pass
  return None


def _traffic_from_profiles():
  """Per-launch DRAM bytes per cell of the stage kernel (ncu)."""
  return _profile_figure('traffic_bytes_per_cell_stage')


# SMs x FP32 lanes per SM of a B200: the FMA-pipe lane rate is this times the
# SM clock.
FP32_LANES = 148 * 128


class ClockSampler:
  """Samples nvidia-smi clocks/throttle reasons in the background."""

  Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
       'clocks_event_reasons.hw_slowdown,'
       'clocks_event_reasons.hw_thermal_slowdown,'
       'clocks_event_reasons.sw_thermal_slowdown,'
       'clocks_event_reasons.sw_power_cap')

  def __init__(self, index: int):
    self.index = index
    self.proc = None
    self.path = None

  def start(self):
    fd, self.path = tempfile.mkstemp(suffix='.csv')
    os.close(fd)
    try:
      self.proc = subprocess.Popen(
          ['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.Q}',
           '--format=csv,noheader,nounits', '-lms', '50'],
          stdout=open(self.path, 'w'), stderr=subprocess.DEVNULL)
    except OSError:
      self.proc = None
      return
    # Start timing only once samples flow (nvidia-smi takes a moment to
    # start), so that the timed region is covered; at most 5 s.
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
      try:
        if os.path.getsize(self.path) > 0:
          break
      except OSError:
        break
      time.sleep(0.02)

  def stop(self):
    if self.proc is None:
      return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unavailable']}
    self.proc.terminate()
    try:
      self.proc.wait(timeout=5)
    except subprocess.TimeoutExpired:
      self.proc.kill()
    sm, smax, reasons = [], [], set()
    names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
             'sw_power_cap']
    with open(self.path) as f:
      for line in f:
        parts = [p.strip() for p in line.split(',')]
        if len(parts) < 9:
          continue
        try:
          sm.append(float(parts[1]))
          smax.append(float(parts[2]))
        except ValueError:
          continue
        for name, val in zip(names, parts[5:9]):
          if val.lower() in ('active', '0x1') or val.startswith('Active'):
            reasons.add(name)
    os.unlink(self.path)
    return {'sm_mhz': statistics.median(sm) if sm else None,
            'sm_max_mhz': max(smax) if smax else None,
            'reasons': sorted(reasons), 'samples': len(sm)}


def _kh_config(n, world):
  """The `config` of the headline workload, shared by both arms."""
  return {'workload': f'kelvin_helmholtz {n}^3 fp32 WENO5+HLLC+viscous, '
                      'SSP-RK3, CFL 0.5, device dt',
          'cells_per_gpu': n ** 3, 'halo_width': 3,
          'parallelism': f'replicas x{world}',
          'l2_flush': f'inputs larger than L2 (5 fields x {n + 6}^3 x 4 B '
                      f'= {5 * (n + 6) ** 3 * 4 / 1e6:.0f} MB per state)',
          'graph': 'one RK3 step captured in a CUDA graph'}


def run_ours(args):
  import torch
  import torch.distributed as dist
  from swirlc_b200 import _native as nat
  from swirlc_b200 import configs, engine
  from swirlc_b200.core import parameter, simulation
  from swirlc_b200.physics import physics_models

  rank, world, local = _env_rank()
  torch.cuda.set_device(local)
  if world > 1:
    dist.init_process_group('nccl', timeout=__import__('datetime').timedelta(seconds=120))
  n = args.n
  user_cfg, state = configs.kelvin_helmholtz(n=n, seed=rank)
  cfg = parameter.SwirlCParameters(user_cfg)
  pm = physics_models.PhysicsModels(cfg)
  dev = torch.device('cuda', local)
  fields = [torch.tensor(state[k], device=dev) for k in
            ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')]
  solver = engine.Solver(cfg, pm, fields[0].shape, torch.float32, dev)
  stepper = engine.Stepper(solver, fields, dt=cfg.dt, cfl=cfg.cfl)
  # Warm-up (eager), then capture one step and warm the graph.
  stepper.step(1)
  torch.cuda.synchronize()
  c0 = nat.launch_count()
  stepper.capture()
  launches_per_step = nat.launch_count() - c0
  stepper.step(max(args.warmup - 1, 1))
  torch.cuda.synchronize()
  cells = n ** 3

  def barrier():
    if world > 1:
      dist.barrier()

  sampler = ClockSampler(local)
  sampler.start()
  barrier()
  torch.cuda.synchronize()
  ev0 = torch.cuda.Event(enable_timing=True)
  ev1 = torch.cuda.Event(enable_timing=True)
  ev0.record()
  stepper.step(args.steps)
  ev1.record()
  torch.cuda.synchronize()
  barrier()
  clocks = sampler.stop()
  ms = ev0.elapsed_time(ev1)
  if world > 1:
    t = torch.tensor([ms], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
  value = world * cells * args.steps / (ms / 1e3)

  # Stage-kernel durations (eager launches bracketed by events on the
  # launching stream), for the roofline of the dominant kernel.
  nstage_steps = 3
  s = solver
  dt = stepper.clock[1:2]
  evs = []
  for _ in range(nstage_steps):
    s.fill_halos(stepper.u)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(); s.stage(stepper.u, None, stepper.w1, nat.SWC_OUT_EULER, dt=dt); b.record()
    evs.append((a, b, 40))
    s.fill_halos(stepper.w1)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(); s.stage(stepper.w1, stepper.u, stepper.w2, nat.SWC_OUT_CONVEX, 0.75, 0.25, dt=dt); b.record()
    evs.append((a, b, 60))
    s.fill_halos(stepper.w2)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(); s.stage(stepper.w2, stepper.u, stepper.u, nat.SWC_OUT_CONVEX, 1 / 3, 2 / 3, dt=dt); b.record()
    evs.append((a, b, 60))
  torch.cuda.synchronize()
  tot_bytes = sum(bpc * cells for _, _, bpc in evs)
  tot_ms = sum(a.elapsed_time(b) for a, b, _ in evs)
  achieved = tot_bytes / (tot_ms / 1e3) / 1e9
  peak, peak_kind = _peaks()
  traffic_pc = _traffic_from_profiles()
  # The bound that holds the stage kernel: its FMA-pipe work (FP32 lane
  # operations per cell and stage, ncu) over the FMA-pipe lane rate at the
  # SM clock sampled during the timed region.
  lane_ops = _profile_figure('fp32_lane_ops_per_cell_stage')
  fp32_pipe = None
  if lane_ops is not None:
    mhz = clocks.get('sm_mhz') or 1965.0
    ach = lane_ops * cells * len(evs) / (tot_ms / 1e3) / 1e12
    pk = FP32_LANES * mhz * 1e6 / 1e12
    fp32_pipe = {'achieved': ach, 'peak': pk, 'unit': 'T lane-ops/s',
                 'frac': ach / pk, 'ops_per_cell_stage': lane_ops,
                 'note': 'FMA-pipe cycles x 128 lanes per SM (an f32x2 '
                         'instruction counts its two lanes); the stage '
                         'kernel is bound here, not by HBM'}

  # End-to-end through the public API: every step copies its input state
  # from pinned host memory, runs Simulation.step and copies the new state
  # back to pinned host memory. The copies run on their own streams (PCIe is
  # full duplex), so step i's compute and read-back overlap step i+1's
  # upload; each step's data dependence (upload -> step -> read-back) is
  # kept by events.
  sim = simulation.Simulation(None, cfg)
  names = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')
  host = {k: torch.from_numpy(state[k]).pin_memory() for k in names}
  host_out = [{k: torch.empty_like(host[k]).pin_memory() for k in names}
              for _ in range(2)]
  replicas = np.array([[[0]]])
  # The same K steps as the device-timed run: the copy pipeline's fill and
  # drain (one upload before the first step, one read-back after the last)
  # are spread over the whole job, as they are for a user's run.
  e2e_steps = max(2, args.steps)
  main = torch.cuda.current_stream()
  up, down = torch.cuda.Stream(), torch.cuda.Stream()

  def e2e_run(nsteps):
    for i in range(nsteps):
      with torch.cuda.stream(up):
        dev_state = {k: host[k].to(dev, non_blocking=True) for k in names}
        loaded = torch.cuda.Event()
        loaded.record(up)
      main.wait_event(loaded)
      for t in dev_state.values():
        t.record_stream(main)
      out = sim.step(0, replicas, 0, dev_state, {})
      done = torch.cuda.Event()
      done.record(main)
      with torch.cuda.stream(down):
        down.wait_event(done)
        for k in names:
          out[k].record_stream(down)
          host_out[i % 2][k].copy_(out[k], non_blocking=True)
    main.wait_stream(down)

  e2e_run(2)
  torch.cuda.synchronize()
  barrier()
  ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  ea.record()
  e2e_run(e2e_steps)
  eb.record()
  torch.cuda.synchronize()
  e2e_ms = ea.elapsed_time(eb)
  if world > 1:
    t = torch.tensor([e2e_ms], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
  state_bytes = sum(host[k].numel() * 4 for k in names)

  cpu = None
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    cpu = cpu_baseline_slabs(n, procs=1, samples=2)

  if rank == 0:
    line = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms / args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic (seeded KH initial condition, configs.kelvin_helmholtz)',
        'config': _kh_config(n, world),
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak,
                     'unit': 'GB/s', 'frac': achieved / peak,
                     'peak_source': peak_kind,
                     'traffic': None if traffic_pc is None else traffic_pc * cells,
                     'kernel': 'stage_kernel (3 launches per step, algorithmic '
                               '40/60/60 B per cell)',
                     'fp32_pipe': fp32_pipe},
        'cpu_baseline': cpu,
        'e2e': {'value': world * cells * e2e_steps / (e2e_ms / 1e3), 'unit': UNIT,
                'h2d_bytes_per_step': state_bytes,
                'd2h_bytes_per_step': state_bytes,
                'api': 'swirlc_b200.core.simulation.Simulation.step',
                'steps': e2e_steps,
                'copies': 'pinned host memory; uploads and read-backs on '
                          'their own streams, overlapping neighbouring '
                          'steps (events order each step\'s upload, step '
                          'and read-back)'},
        'gpu_launches': launches_per_step * args.steps,
        'clocks': clocks,
    }
    print(json.dumps(line), flush=True)
  del stepper.graph
  if world > 1:
    dist.destroy_process_group()


def run_decomposed(args):
  """One Kelvin-Helmholtz domain of --n^3 cells split into the cx x cy x cz
  blocks of --decomposed (strong scaling): one block per rank over
  torch.distributed (NCCL) when launched with cx*cy*cz ranks, else every
  block in this process (LocalExchange). With NCCL (or --overlap) the halo
  updates overlap the inner boxes' stage work
  (decomposition.DecomposedStepper); --no-overlap turns that off."""
  import torch
  import torch.distributed as dist
  from swirlc_b200 import configs, decomposition
  rank, world, local = _env_rank()
  torch.cuda.set_device(local)
  shape = tuple(int(v) for v in args.decomposed.split(','))
  if len(shape) != 3:
    raise SystemExit('--decomposed takes cx,cy,cz')
  nblk = int(np.prod(shape))
  if world > 1:
    if nblk != world:
      raise SystemExit(f'--decomposed {args.decomposed} needs {nblk} ranks')
    dist.init_process_group(
        'nccl', timeout=__import__('datetime').timedelta(seconds=120))
  n = args.n
  user_cfg, state = configs.kelvin_helmholtz(n=n)
  user_cfg = dict(user_cfg, cx=shape[0], cy=shape[1], cz=shape[2])
  replicas = np.arange(nblk).reshape(shape)
  blocks = decomposition.split_state(state, replicas, 3)
  del state
  mine = {rank: blocks[rank]} if world > 1 else blocks
  ds = decomposition.DecomposedStepper(
      user_cfg, mine, transport='dist' if world > 1 else 'local',
      overlap=False if args.no_overlap else (True if args.overlap else None))
  ds.step(args.warmup)
  torch.cuda.synchronize()

  def barrier():
    if world > 1:
      dist.barrier()

  sampler = ClockSampler(local)
  sampler.start()
  barrier()
  torch.cuda.synchronize()
  e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
  e0.record()
  ds.step(args.steps)
  e1.record()
  torch.cuda.synchronize()
  barrier()
  clocks = sampler.stop()
  ms = e0.elapsed_time(e1)
  if world > 1:
    t = torch.tensor([ms], device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
  if rank == 0:
    line = {
        'metric': f'RK3 cell-updates/s, one {n}^3 domain decomposed',
        'value': n ** 3 * args.steps / (ms / 1e3), 'unit': UNIT,
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms / args.steps, 'higher_is_better': True,
        'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic (seeded KH initial condition, configs.kelvin_helmholtz)',
        'config': {'workload': f'kelvin_helmholtz {n}^3 fp32 WENO5+HLLC+'
                               'viscous, SSP-RK3, CFL 0.5, device dt',
                   'blocks': list(shape),
                   'transport': 'nccl' if world > 1 else 'local',
                   'overlap': ds.overlap,
                   'l2_flush': 'inputs larger than L2'},
        'clocks': clocks,
    }
    print(json.dumps(line), flush=True)
  if world > 1:
    dist.destroy_process_group()


BATCH_METRIC = ('RK3 cell-updates/s, 64 batched quasi-1-D Riemann problems '
                'fp32 WENO5+HLLC, per-member CFL dt')


def _plain_rate(configs, engine, parameter, physics_models, user_cfg, state,
                steps):
  """cell-updates/s of the single-grid step (one-step CUDA graph)."""
  import torch
  cfg = parameter.SwirlCParameters(user_cfg)
  s = engine.Solver(cfg, physics_models.PhysicsModels(cfg), state['rho'].shape)
  f = [torch.tensor(state[k], device='cuda') for k in
       ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')]
  st = engine.Stepper(s, f, dt=cfg.dt, cfl=cfg.cfl)
  st.step(1)
  st.capture()
  st.step(3)
  a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  torch.cuda.synchronize()
  a.record()
  st.step(steps)
  b.record()
  torch.cuda.synchronize()
  return s.nx * s.ny * s.nz * steps / (a.elapsed_time(b) / 1e3)


def _batch_cpu_sample(members, procs: int = 1):
  """CPU oracle: one SSP-RK3 step of each of the members (float32)."""
  import multiprocessing as mp
  from oracle import swirlc_oracle as orc
  keys = ('halo_width', 'dx', 'dy', 'dz', 'interpolation_scheme',
          'numeric_flux_scheme', 'include_diffusion', 'transport_parameters',
          'x', 'y', 'z', 'bc', 'dt')
  work, cells = [], 0
  for cfg, state in members:
    ocfg = orc.make_cfg(**{k: cfg[k] for k in keys if k in cfg})
    work.append((ocfg, {k: np.asarray(v, np.float32) for k, v in state.items()}))
    cells += cfg['nx'] * cfg['ny'] * cfg['nz']
  t0 = time.perf_counter()
  if procs <= 1:
    for w in work:
      _oracle_rk3_worker(w)
  else:
    with mp.get_context('spawn').Pool(procs) as pool:
      pool.map(_oracle_rk3_worker, work)
  secs = time.perf_counter() - t0
  return cells / secs, secs, cells


def _batch_sample_members(configs):
  return [m for m in configs.riemann_batch() if m[0]['nx'] * m[0]['ny'] *
          m[0]['nz'] <= 120000]


def run_batch(args):
  """The 64-member Riemann batch (configs.riemann_batch) stepped by
  swc_batch_step under a CUDA graph; each rank runs its own batch (seed =
  rank)."""
  import torch
  import torch.distributed as dist
  from swirlc_b200 import _native as nat
  from swirlc_b200 import batch, configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models

  rank, world, local = _env_rank()
  torch.cuda.set_device(local)
  if world > 1:
    dist.init_process_group('nccl', timeout=__import__('datetime').timedelta(seconds=120))
  members = configs.riemann_batch(seed=rank)
  bs = batch.BatchStepper(members)
  cells = bs.cells()
  bs.step(1)
  tune = bs.autotune(steps=2, reps=2)
  torch.cuda.synchronize()
  c0 = nat.launch_count()
  bs.capture(steps=1)
  launches_per_step = nat.launch_count() - c0
  bs.step(max(args.warmup - 1, 1))
  torch.cuda.synchronize()

  def barrier():
    if world > 1:
      dist.barrier()

  sampler = ClockSampler(local)
  sampler.start()
  barrier()
  torch.cuda.synchronize()
  ev0, ev1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
  ev0.record()
  bs.step(args.steps)
  ev1.record()
  torch.cuda.synchronize()
  barrier()
  clocks = sampler.stop()
  ms = ev0.elapsed_time(ev1)
  if world > 1:
    t = torch.tensor([ms], device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
  value = world * cells * args.steps / (ms / 1e3)
  bs.graph = None

  # Reference points on this GPU: the members one after another, and the
  # plain single-grid kernel on large grids of the same scheme.
  seq = batch.sequential_plain(members, args.steps)
  sod_cfg, sod_state = configs.sod(n=4096, ny=32, nz=32)
  plain_thin = _plain_rate(configs, engine, parameter, physics_models,
                           dict(sod_cfg, t_end=0.0), sod_state, args.steps)
  kh_cfg, kh_state = configs.kelvin_helmholtz(n=256)
  plain_cube = _plain_rate(configs, engine, parameter, physics_models,
                           dict(kh_cfg, include_diffusion=False), kh_state,
                           max(5, args.steps // 2))

  # End to end: every member's state from pinned host memory, one batch
  # step, every member's state back to pinned host memory.
  names = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')
  host = [[torch.from_numpy(np.ascontiguousarray(st[k], np.float32)).pin_memory()
           for k in names] for _, st in members]
  back = [[torch.empty_like(h).pin_memory() for h in hs] for hs in host]
  e2e_steps = max(1, min(args.steps, 5))

  def e2e_once():
    for u, hs in zip(bs.u, host):
      for f, h in zip(u, hs):
        f.copy_(h, non_blocking=True)
    bs.step(1)
    for u, hs in zip(bs.u, back):
      for f, h in zip(u, hs):
        h.copy_(f, non_blocking=True)

  e2e_once()
  torch.cuda.synchronize()
  barrier()
  ea, eb = (torch.cuda.Event(enable_timing=True) for _ in range(2))
  ea.record()
  for _ in range(e2e_steps):
    e2e_once()
  eb.record()
  torch.cuda.synchronize()
  e2e_ms = ea.elapsed_time(eb)
  if world > 1:
    t = torch.tensor([e2e_ms], device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
  state_bytes = sum(h.numel() * 4 for hs in host for h in hs)

  cpu = None
  if rank == 0 and world == 1 and not args.no_cpu_baseline:
    sample = _batch_sample_members(configs)
    rate, secs, scells = _batch_cpu_sample(sample)
    cpu = {'value': rate, 'unit': UNIT, 'cores': 1, 'kind': 'port',
           'sample': f'one SSP-RK3 step of the {len(sample)} members with '
                     f'<= 120k cells ({scells} cells), NumPy float32 oracle, '
                     f'{secs:.1f} s'}
  peak, peak_kind = _peaks()
  achieved = ALG_BYTES_PER_CELL_UPDATE * cells * args.steps / (ms / 1e3) / 1e9
  if rank == 0:
    line = {
        'metric': BATCH_METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms / args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic (seeded members, configs.riemann_batch)',
        'config': {'workload': 'riemann_batch: 64 members, nx log-uniform '
                               '[64, 4096], ny = nz in {4, 8, 16, 32}, '
                               'WENO5+HLLC, SSP-RK3, CFL 0.5 per member',
                   'cells_per_gpu': cells, 'members': bs.n_members,
                   'parallelism': f'replicas x{world}',
                   'l2_flush': 'inputs larger than L2 (3 states x 5 fields '
                               'of all members = 1.9 GB)',
                   'graph': 'one batch step captured in a CUDA graph',
                   'autotune': {'small_ny': tune['small_ny'],
                                'zseg': tune['zseg']}},
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak,
                     'unit': 'GB/s', 'frac': achieved / peak,
                     'peak_source': peak_kind, 'traffic': None,
                     'kernel': 'whole batch step (stage_batch_kernel + '
                               'halo_batch_kernel), algorithmic 160 B per '
                               'cell-update'},
        'plain_kernel': {'sod_4096x32x32': plain_thin,
                         'kh_256^3_inviscid': plain_cube,
                         'batch_over_kh256': value / world / plain_cube,
                         'batch_over_same_shape': value / world / plain_thin},
        'sequential_members': {'value': seq['cell_updates_per_s'], 'unit': UNIT,
                               'how': 'each member its own one-step graph, '
                                      'members one after another'},
        'cpu_baseline': cpu,
        'e2e': {'value': world * cells * e2e_steps / (e2e_ms / 1e3), 'unit': UNIT,
                'h2d_bytes_per_step': state_bytes,
                'd2h_bytes_per_step': state_bytes,
                'api': 'swirlc_b200.batch.BatchStepper.step'},
        'gpu_launches': launches_per_step * args.steps,
        'clocks': clocks,
    }
    print(json.dumps(line), flush=True)
  if world > 1:
    dist.destroy_process_group()


ADJ_METRIC = ('adjoint/forward time ratio, KH 128^3 fp32 WENO5+HLLC+viscous, '
              '200 SSP-RK3 steps, checkpoints every 20')


def _adjoint_fd_check(n, steps, k, ndir=16, hs=(1e-6,), offset=0.0):
  """Float64 central differences of the vorticity energy along seeded random
  directions in (initial velocity, nu), against the adjoint gradient, at
  each step size in `hs` (the same directions for every h).

  The scheme is not everywhere differentiable. min/max wave speeds and
  HLLC's branch selection are kinks: a central difference straddling one
  errs in proportion to h. HLLC's cut-off s_m = 0 for |s_m| < 1e-6
  (hllc.py:328-341) is a jump: a difference straddles one with probability
  proportional to h but then errs by jump / h, an error floor that does not
  fall with h. `offset` adds a uniform velocity to the initial state (a
  Galilean shift of the periodic flow), which keeps the contact speeds of
  most faces away from that cut-off."""
  import torch
  from swirlc_b200 import adjoint, configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  user_cfg, state = configs.kelvin_helmholtz(n=n, dtype=np.float64)
  cfg = parameter.SwirlCParameters(user_cfg)
  names = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')
  f = [torch.tensor(state[k_], dtype=torch.float64, device='cuda') for k_ in names]
  s = engine.Solver(cfg, physics_models.PhysicsModels(cfg), f[0].shape,
                    torch.float64)
  hw = s.hw
  inner = (slice(hw, -hw),) * 3
  rho = f[0]
  # Control: the initial velocity (its seeded perturbation included) at
  # fixed rho and p.
  vel = [f[i] / rho for i in (1, 2, 3)]
  p0 = 0.4 * (f[4] - 0.5 * rho * (vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2))
  vel = [x + offset for x in vel]

  def state_of(v):
    ke = 0.5 * rho * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
    return [rho, rho * v[0], rho * v[1], rho * v[2], p0 / 0.4 + ke]

  st = engine.Stepper(s, [x.clone() for x in state_of(vel)], dt=cfg.dt,
                      cfl=cfg.cfl)
  dts = []
  for _ in range(steps):
    st.step(1)
    dts.append(float(st.clock[1].item()))
  del st

  def loss(out):
    return adjoint.vorticity_energy(out, hw, s.grid.dx, s.grid.dy, s.grid.dz)

  nu0 = float(s.scheme.nu)
  run = adjoint.RunAdjoint(s, checkpoint_every=k)
  v = [x.clone().requires_grad_(True) for x in vel]
  nu = torch.tensor(nu0, dtype=torch.float64, requires_grad=True)
  out = adjoint.simulate(run, state_of(v), dts, nu)
  j = loss(out)
  j.backward()
  gv = [x.grad for x in v]
  gnu = float(nu.grad)
  rng = np.random.default_rng(0)
  rels = {h: [] for h in hs}
  for _ in range(ndir):
    d = []
    for x in vel:
      dd = torch.zeros_like(x)
      dd[inner] = torch.tensor(rng.standard_normal(x[inner].shape), dtype=x.dtype,
                               device='cuda')
      d.append(dd)
    dnu = float(rng.standard_normal()) * nu0
    ad = sum(float((g[inner] * b[inner]).sum()) for g, b in zip(gv, d)) + gnu * dnu
    for h in hs:
      js = []
      for sgn in (1.0, -1.0):
        s.scheme.nu = nu0 + sgn * h * dnu
        r2 = adjoint.RunAdjoint(s, checkpoint_every=k)
        o2 = r2.run(state_of([a + sgn * h * b for a, b in zip(vel, d)]), dts)
        js.append(float(loss(o2)))
      s.scheme.nu = nu0
      fd = (js[0] - js[1]) / (2 * h)
      rels[h].append(abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
  per_h = [{'h': h, 'median_rel_err': float(np.median(rels[h])),
            'max_rel_err': float(np.max(rels[h]))} for h in hs]
  res = {'directions': ndir, 'dtype': 'f64', 'grid': f'{n}^3',
         'steps': steps, 'loss': float(j.detach()), 'velocity_offset': offset}
  res.update(per_h[-1])
  if len(hs) > 1:
    res['by_h'] = per_h
  return res


def run_adjoint(args):
  """Config 5: the discrete adjoint of 200 KH steps at 128^3 (fp32)."""
  import torch
  from swirlc_b200 import _native as nat
  from swirlc_b200 import adjoint, configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  rank, world, local = _env_rank()
  torch.cuda.set_device(local)
  n, steps, k = args.adj_n, args.adj_steps, 20
  user_cfg, state = configs.kelvin_helmholtz(n=n, seed=rank)
  cfg = parameter.SwirlCParameters(user_cfg)
  names = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')
  f = [torch.tensor(state[k_], device='cuda') for k_ in names]
  s = engine.Solver(cfg, physics_models.PhysicsModels(cfg), f[0].shape,
                    torch.float32)
  st = engine.Stepper(s, [x.clone() for x in f], dt=cfg.dt, cfl=cfg.cfl)
  dts = []
  for _ in range(steps):
    st.step(1)
    dts.append(float(st.clock[1].item()))
  del st
  run = adjoint.RunAdjoint(s, checkpoint_every=k, steps=steps)

  def loss(out):
    return adjoint.vorticity_energy(out, s.hw, s.grid.dx, s.grid.dy, s.grid.dz)

  def loss_grad(out):
    x = [o.detach().clone().requires_grad_(True) for o in out]
    g = torch.autograd.grad(loss(x), x, allow_unused=True)
    return [torch.zeros_like(o) if gi is None else gi for o, gi in zip(out, g)]

  # Warm-up on a short run (kernel variants loaded, allocator warm).
  for _ in range(max(1, args.warmup - 2)):
    o0 = run.run(f, dts[:k])
    run.backward(loss_grad(o0))
  torch.cuda.synchronize()
  sampler = ClockSampler(local)
  sampler.start()
  # Three timed forward runs + sweeps; the line reports the median ratio
  # (the sweeps' spread from run to run is in `repeats`).
  reps = []
  for _ in range(3):
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    out = run.run(f, dts)
    e[1].record()
    c0 = nat.launch_count()
    g_in, nub = run.backward(loss_grad(out))
    e[2].record()
    torch.cuda.synchronize()
    launches = nat.launch_count() - c0
    reps.append((e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])))
  clocks = sampler.stop()
  fwd_ms, bwd_ms = sorted(reps, key=lambda r: r[1] / r[0])[1]
  cells = n ** 3
  # The same run keeping every stage state (no recomputation in the sweep).
  del run
  torch.cuda.empty_cache()
  run_all = adjoint.RunAdjoint(s, checkpoint_every=0, steps=steps)
  e2 = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
  e2[0].record()
  out_all = run_all.run(f, dts)
  e2[1].record()
  run_all.backward(loss_grad(out_all))
  e2[2].record()
  torch.cuda.synchronize()
  fwd_all, bwd_all = e2[0].elapsed_time(e2[1]), e2[1].elapsed_time(e2[2])
  del run_all, out_all
  torch.cuda.empty_cache()
  hs = tuple(float(x) for x in args.fd_h.split(','))
  fd = _adjoint_fd_check(n, steps, k, hs=hs) if args.fd_check else None
  if fd is not None and args.fd_offset:
    fd['galilean_shift'] = _adjoint_fd_check(n, steps, k, hs=hs,
                                             offset=args.fd_offset)
  if rank == 0:
    line = {
        'metric': ADJ_METRIC, 'value': bwd_ms / fwd_ms, 'unit': 'ratio',
        'n_gpus': world, 'steps': steps, 'warmup': args.warmup,
        'ms_per_step': bwd_ms / steps, 'higher_is_better': False,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic (seeded KH initial condition)',
        'config': {'workload': f'kelvin_helmholtz {n}^3 fp32 WENO5+HLLC+viscous '
                               f'nu=1e-4, {steps} SSP-RK3 steps (device-CFL '
                               'dt sequence, held fixed), checkpoints every '
                               f'{k}, loss = vorticity energy',
                   'cells': cells, 'l2_flush': 'inputs larger than L2'},
        'forward_ms': fwd_ms, 'backward_ms': bwd_ms,
        'repeats': [{'forward_ms': a, 'backward_ms': b, 'ratio': b / a}
                    for a, b in reps],
        'forward_cell_updates_per_s': cells * steps / (fwd_ms / 1e3),
        'target': 'backward <= 3 x forward',
        'stored_stages': {'forward_ms': fwd_all, 'backward_ms': bwd_all,
                          'ratio': bwd_all / fwd_all,
                          'how': 'checkpoint_every=0: every stage state kept '
                                 f'({steps} x 3 states, buffers allocated '
                                 'once by the runner, no recomputation)'},
        'grad_nu': nub,
        'gpu_launches_backward': launches,
        'fd_check': fd,
        'clocks': clocks,
    }
    print(json.dumps(line), flush=True)


def _graph_steps(user_cfg, state, steps, warmup, dtype_name='f32'):
  """Steps of the single-grid path replayed from a one-step CUDA graph:
  (ms per step, the stepper). `warmup` steps run first on a throw-away copy
  of the state, so that the timed run starts from the initial state."""
  import torch
  from swirlc_b200 import engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  dtype = torch.float32 if dtype_name == 'f32' else torch.float64
  cfg = parameter.SwirlCParameters(user_cfg)
  s = None

  def stepper():
    nonlocal s
    f = [torch.tensor(state[k], dtype=dtype, device='cuda') for k in
         ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')]
    if s is None:
      s = engine.Solver(cfg, physics_models.PhysicsModels(cfg), f[0].shape,
                        dtype)
    st = engine.Stepper(s, f, dt=cfg.dt, cfl=cfg.cfl, t_end=cfg.t_end,
                        scheme=cfg.time_integration_scheme)
    st.capture()
    return st

  warm = stepper()
  warm.step(warmup)
  del warm
  st = stepper()
  torch.cuda.synchronize()
  e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
  e0.record()
  st.step(steps)
  e1.record()
  torch.cuda.synchronize()
  return e0.elapsed_time(e1) / steps, st


def run_config_case(args):
  """Config 1 (Sod 256x8x8 to t = 0.2) or config 3 (buoyant bubble
  512x512x256, 50 steps): time per step under a CUDA graph and the float32
  error against the same kernels in float64."""
  import torch
  from swirlc_b200 import accuracy, configs
  if args.workload == 'sod':
    user_cfg, state = configs.sod()
    # Step count to t = 0.2 from a float64 run (its dt sequence is also the
    # one the error report replays).
    rep = accuracy.report('sod', user_cfg, state, 100000)
    steps = rep['steps']
    name = 'sod 256x8x8 fp32 WENO5+HLLC, CFL 0.5 to t = 0.2'
  else:
    user_cfg, state = configs.buoyant_bubble()
    steps = 50
    rep = accuracy.report('bubble', user_cfg, state, steps)
    name = ('buoyant bubble 512x512x256 fp32 MUSCL(van Leer)+HLL, gravity, '
            'Dirichlet/Neumann z walls, 50 steps, CFL 0.2')
  sampler = ClockSampler(0)
  sampler.start()
  warmup = max(3, args.warmup)
  ms, st = _graph_steps(user_cfg, state, steps, warmup)
  clocks = sampler.stop()
  s = st.s
  cells = s.nx * s.ny * s.nz
  line = {
      'metric': f'{args.workload}: ms per SSP-RK3 step (CUDA graph) and '
                'float32 error vs float64',
      'value': ms, 'unit': 'ms/step', 'n_gpus': 1, 'steps': steps,
      'warmup': warmup, 'ms_per_step': ms, 'higher_is_better': False,
      'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
      'data': 'synthetic (configs.' + ('sod' if args.workload == 'sod'
                                       else 'buoyant_bubble') + ')',
      'config': {'workload': name, 'cells': cells,
                 'l2': ('state resident in L2 (16k cells; time to solution)'
                        if args.workload == 'sod' else
                        'inputs larger than L2 (1.3 GB of fields)')},
      'time_to_solution_ms': ms * steps,
      'cell_updates_per_s': cells / (ms / 1e3),
      'fp64_error': rep,
      'clocks': clocks,
  }
  print(json.dumps(line), flush=True)


def run_profile(args):
  """Eager RK3 steps of the workload, no timing: the command ncu captures.
  kh256: Kelvin-Helmholtz at --n^3; bubble: the buoyant bubble at
  --n x --n x --n/2 (its 2:2:1 shape)."""
  import torch
  from swirlc_b200 import configs, engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  if args.workload == 'bubble':
    user_cfg, state = configs.buoyant_bubble(nx=args.n, ny=args.n,
                                             nz=args.n // 2)
  else:
    user_cfg, state = configs.kelvin_helmholtz(n=args.n)
  cfg = parameter.SwirlCParameters(user_cfg)
  pm = physics_models.PhysicsModels(cfg)
  fields = [torch.tensor(state[k], device='cuda') for k in
            ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')]
  solver = engine.Solver(cfg, pm, fields[0].shape, torch.float32)
  stepper = engine.Stepper(solver, fields, dt=cfg.dt, cfl=cfg.cfl)
  stepper.step(args.profile_steps)
  torch.cuda.synchronize()


def _oracle_rk3_worker(payload):
  from oracle import swirlc_oracle as orc
  cfg, state = payload
  t0 = time.perf_counter()
  orc.rk3(state, cfg.dt, lambda s: orc.rhs(s, cfg))
  return time.perf_counter() - t0


# One host process steps, per sample, SLAB_PLANES z planes x SLAB_X x-rows
# of the 256^3 grid (all y): about 2-3 s of NumPy work, so that a reference
# run of 50 samples stays within a few minutes.
SLAB_PLANES = 8
SLAB_X = 64


class KHSlabSampler:
  """Times the CPU oracle (the NumPy float32 restatement of the reference
  path) on blocks of the n^3 Kelvin-Helmholtz state.

  One sample step: `procs` host processes each take one SSP-RK3 step of a
  block of SLAB_PLANES interior z planes x SLAB_X interior x rows x all n y
  columns, plus 3 halo layers on each side of every axis (the oracle
  evaluates its halo layers too, so the rate counts interior cell-updates
  only and is conservative); successive samples move through the domain.
  The pool is started with `spawn` before any work.
  """

  def __init__(self, n: int, procs: int):
    import multiprocessing as mp
    from swirlc_b200 import configs
    from oracle import swirlc_oracle as orc
    self.n = n
    self.sx = min(SLAB_X, n)
    self.sz = min(SLAB_PLANES, n)
    self.blocks = (n // self.sz) * (n // self.sx)
    self.procs = max(1, min(procs, self.blocks))
    user_cfg, self.state = configs.kelvin_helmholtz(n=n)
    keys = ('halo_width', 'dx', 'dy', 'dz', 'interpolation_scheme',
            'numeric_flux_scheme', 'include_diffusion',
            'transport_parameters', 'x', 'y', 'dt')
    self.cfg = orc.make_cfg(**{k: user_cfg[k] for k in keys})
    self.cfg.bc = orc.periodic_bc()
    self.hw = user_cfg['halo_width']
    self.pool = (mp.get_context('spawn').Pool(self.procs)
                 if self.procs > 1 else None)
    self.cells = self.procs * self.sz * self.sx * n

  def _slab(self, b: int):
    nzb = self.n // self.sz
    z0, x0 = (b % nzb) * self.sz, (b // nzb) * self.sx
    iz = np.arange(z0, z0 + self.sz + 2 * self.hw) % self.n + self.hw
    ix = np.arange(x0, x0 + self.sx + 2 * self.hw) % self.n + self.hw
    return {k: np.ascontiguousarray(v[iz][:, ix]) for k, v in self.state.items()}

  def step(self, j: int) -> float:
    """Wall seconds of sample step j."""
    tasks = [(self.cfg, self._slab((j * self.procs + p) % self.blocks))
             for p in range(self.procs)]
    t0 = time.perf_counter()
    if self.pool is None:
      _oracle_rk3_worker(tasks[0])
    else:
      self.pool.map(_oracle_rk3_worker, tasks)
    return time.perf_counter() - t0

  def describe(self) -> str:
    return (f'one SSP-RK3 step of {self.procs} block(s) of {self.sz} z '
            f'planes x {self.sx} x-rows x {self.n} (+3 halo layers a side) '
            f'of the KH {self.n}^3 state per sample, NumPy float32 oracle, '
            f'{self.procs} process(es)')

  def close(self):
    if self.pool is not None:
      self.pool.close()
      self.pool.join()


def cpu_baseline_slabs(n: int, procs: int = 1, samples: int = 2):
  """The cpu_baseline object: the oracle on `samples` slab steps."""
  sampler = KHSlabSampler(n, procs)
  try:
    secs = [sampler.step(j) for j in range(samples)]
  finally:
    sampler.close()
  v = sampler.cells * len(secs) / sum(secs)
  return {'value': v, 'unit': UNIT, 'cores': sampler.procs, 'kind': 'port',
          'sample': sampler.describe() + f', {sum(secs):.1f} s wall'}


def run_reference_batch(args):
  from swirlc_b200 import configs
  procs = os.cpu_count() or 1
  sample = _batch_sample_members(configs)
  rates = []
  for _ in range(max(1, min(args.steps, 3))):
    rate, secs, scells = _batch_cpu_sample(sample, procs)
    rates.append(rate)
  v = statistics.median(rates)
  desc = (f'one SSP-RK3 step of the {len(sample)} members with <= 120k cells '
          f'({scells} cells) over {procs} processes, NumPy float32 oracle')
  line = {
      'impl': 'reference', 'metric': BATCH_METRIC, 'value': v, 'unit': UNIT,
      'n_gpus': int(os.environ.get('WORLD_SIZE', '1')), 'steps': args.steps,
      'warmup': args.warmup, 'ms_per_step': scells / v * 1e3,
      'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
      'dtype': 'f32', 'data': 'synthetic (seeded members)',
      'config': {'workload': 'riemann_batch (CPU sample)',
                 'parallelism': f'{procs} host processes'},
      'cpu_baseline': {'value': v, 'unit': UNIT, 'cores': procs,
                       'kind': 'port', 'sample': desc},
      'e2e': {'value': v, 'unit': UNIT, 'h2d_bytes_per_step': 0,
              'd2h_bytes_per_step': 0},
  }
  print(json.dumps(line), flush=True)


def run_reference(args):
  """The reference arm: the CPU oracle on this host's cores, W warm-up and
  K timed sample steps (KHSlabSampler), on the headline workload's config.
  The reference's own TensorFlow path needs TensorFlow and swirl_lm, which
  are not installed (no network); the oracle restates it."""
  rank, world, _ = _env_rank()
  if rank != 0:
    return
  if args.workload == 'riemann_batch':
    run_reference_batch(args)
    return
  try:
    procs = len(os.sched_getaffinity(0))
  except AttributeError:
    procs = os.cpu_count() or 1
  sampler = KHSlabSampler(args.n, procs)
  try:
    for j in range(args.warmup):
      sampler.step(j)
    secs = [sampler.step(args.warmup + j) for j in range(args.steps)]
  finally:
    sampler.close()
  t = sum(secs)
  v = sampler.cells * args.steps / t
  line = {
      'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': UNIT,
      'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
      'ms_per_step': t / args.steps * 1e3, 'higher_is_better': True,
      'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
      'data': 'synthetic (seeded KH initial condition, configs.kelvin_helmholtz)',
      'config': _kh_config(args.n, world),
      'cpu_baseline': {'value': v, 'unit': UNIT, 'cores': sampler.procs,
                       'kind': 'port',
                       'sample': sampler.describe() + '; a step of this '
                                 f'line is one sample ({sampler.cells} '
                                 'interior cell-updates)'},
      'e2e': {'value': v, 'unit': UNIT, 'h2d_bytes_per_step': 0,
              'd2h_bytes_per_step': 0},
      'note': 'the reference TensorFlow path needs TensorFlow and swirl_lm, '
              'which are not installed; the NumPy oracle restating it runs',
  }
  print(json.dumps(line), flush=True)


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--gpus', type=int, default=1)
  ap.add_argument('--steps', type=int, default=50)
  ap.add_argument('--warmup', type=int, default=3)
  ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
  ap.add_argument('--n', type=int, default=N_CELLS_EDGE)
  ap.add_argument('--no-cpu-baseline', action='store_true')
  ap.add_argument('--adj-n', type=int, default=128)
  ap.add_argument('--adj-steps', type=int, default=200)
  ap.add_argument('--fd-check', action='store_true',
                  help='adjoint workload: add the float64 16-direction '
                       'central-difference check at full size')
  ap.add_argument('--fd-offset', type=float, default=0.0,
                  help='--fd-check: repeat the check on the flow shifted by '
                       'this uniform velocity in x, y and z')
  ap.add_argument('--fd-h', default='1e-6',
                  help='comma-separated central-difference steps of '
                       '--fd-check (the last one is the reported figure)')
  ap.add_argument('--workload', default='kh256',
                  choices=['kh256', 'riemann_batch', 'adjoint', 'sod',
                           'bubble'],
                  help='kh256: the headline 256^3 Kelvin-Helmholtz step; '
                       'riemann_batch: 64 batched Riemann problems')
  ap.add_argument('--decomposed', default='',
                  help='cx,cy,cz: one --n^3 domain split into blocks (one '
                       'per rank under torchrun, else all in this process)')
  ap.add_argument('--no-overlap', action='store_true',
                  help='--decomposed: halo update before each stage instead '
                       'of behind the inner boxes')
  ap.add_argument('--overlap', action='store_true',
                  help='--decomposed: halo update behind the inner boxes '
                       'also with all blocks in this process (by default '
                       'only the NCCL transport overlaps)')
  ap.add_argument('--profile-steps', type=int, default=0,
                  help='only run this many eager RK3 steps of the workload '
                       '(a small, untimed command for ncu captures)')
  args = ap.parse_args()
  if args.profile_steps:
    run_profile(args)
    return
  if args.warmup < 3:
    args.warmup = 3
  if args.impl == 'reference':
    run_reference(args)
  elif args.decomposed:
    run_decomposed(args)
  elif args.workload == 'riemann_batch':
    run_batch(args)
  elif args.workload == 'adjoint':
    run_adjoint(args)
  elif args.workload in ('sod', 'bubble'):
    run_config_case(args)
  else:
    run_ours(args)


if __name__ == '__main__':
  main()
