"""Device-side domain description and the fused step loop.

`Solver` turns a reference config (`SwirlCParameters`) plus the shape and
dtype of one replica's fields into the C-ABI descriptors (SwcGrid, SwcScheme,
SwcFieldBC) and issues the kernels of libswirlc_b200.so on the current torch
CUDA stream. `Stepper` owns the work buffers and the device clock of a
time loop and can capture one step in a CUDA graph.

Fields are torch CUDA tensors in the reference layout [nz+2h, nx+2h, ny+2h]
(y contiguous), halos included, ordered rho, rho_u, rho_v, rho_w, rho_e.
"""

from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from swirlc_b200 import _native as nat
from swirlc_b200.boundary import bc_types
from swirlc_b200.common import types
from swirlc_b200.common import utils
from swirlc_b200.physics import constant

_INTERP = {'WENO_5': nat.SWC_WENO5, 'WENO_3': nat.SWC_WENO3,
           'MUSCL': nat.SWC_MUSCL, 'NODE': nat.SWC_NODE}
_LIMITER = {'van_leer': nat.SWC_LIM_VAN_LEER, 'mc': nat.SWC_LIM_MC,
            'minmod': nat.SWC_LIM_MINMOD, 'minmod3': nat.SWC_LIM_MINMOD3}
_CELL_AVG = bc_types.BoundaryDictionaryType.CELL_AVERAGES.value
_CELL_FACE = bc_types.BoundaryDictionaryType.CELL_FACES.value
_CELL_FLUX = bc_types.BoundaryDictionaryType.INTERCELL_FLUXES.value


def interp_code(cfg) -> int:
  """Scheme code; errors as compressible_navier_stokes.py:581-595."""
  scheme = getattr(cfg, 'interpolation_scheme', None)
  if scheme not in _INTERP:
    raise NotImplementedError(
        f'"{scheme}" is not implemented as an "interpolation_scheme". Valid '
        "options are: ['WENO_3', 'WENO_5', 'MUSCL']")
  return _INTERP[scheme]


def riemann_code(cfg) -> int:
  """Flux code; errors as riemann_solver.py:53-62."""
  scheme = getattr(cfg, 'numeric_flux_scheme', None)
  if scheme == 'HLL':
    return nat.SWC_HLL
  if scheme == 'HLLC':
    return nat.SWC_HLLC
  raise ValueError(
      f'"{scheme}" is not implemented as a "numeric_flux_scheme". Valid '
      "options are: ['HLL', 'HLLC']")


def _plane(val, dim: int, shape3: Sequence[int], dtype, device) -> torch.Tensor:
  """A Dirichlet layer value as a [A, B] plane (see SwcBC.planes)."""
  nz, nx, ny = shape3
  ab = {0: (nz, ny), 1: (nz, nx), 2: (nx, ny)}[dim]
  if isinstance(val, (int, float, np.floating, np.integer)):
    return torch.full(ab, float(val), dtype=dtype, device=device)
  if isinstance(val, (list, tuple)):
    t = torch.stack([torch.as_tensor(np.asarray(
        v.cpu() if isinstance(v, torch.Tensor) else v)) for v in val])
  else:
    t = torch.as_tensor(np.asarray(val.cpu() if isinstance(val, torch.Tensor)
                                   else val))
  t = t.to(dtype=dtype).reshape(ab).to(device)
  return t.contiguous()


def fill_field_bc(fbc, spec, via: int, shape3, hw: int, dtype, device,
                  name: str = '') -> list:
  """Fills one SwcFieldBC from a reference per-variable BC dict
  {dim: {0: (type, value), 1: (type, value)}} (bc_types.BCDict).

  Returns the device tensors that back per-layer Dirichlet planes; keep them
  alive while the descriptor is in use.
  """
  keep = []
  fbc.via_primitive = via
  for di, dim in enumerate(types.DIMS):
    sides = spec.get(dim) if isinstance(spec, dict) else None
    if not sides:
      for s in range(2):
        fbc.side[di][s].kind = nat.SWC_BC_NONE
      continue
    # A PERIODIC entry makes the dim periodic (boundary.py:65-68).
    periodic = any(bc_types.bc_value(sides[s][0]) == 0 for s in (0, 1)
                   if s in sides)
    for s in range(2):
      b = fbc.side[di][s]
      if periodic:
        b.kind = nat.SWC_BC_PERIODIC
        continue
      kind = bc_types.bc_value(sides[s][0])
      val = sides[s][1] if len(sides[s]) > 1 else 0.0
      if kind == bc_types.BoundaryCondition.DIRICHLET.value:
        b.kind = nat.SWC_BC_DIRICHLET
        if isinstance(val, (list, tuple)):
          layers = [_plane(v, di, shape3, dtype, device) for v in val]
          if len(layers) != hw:
            raise ValueError(
                f'Dirichlet BC for {name} along {dim} has {len(layers)} '
                f'layers; halo_width is {hw}.')
          planes = torch.stack(layers).contiguous()
          keep.append(planes)
          b.per_layer = 1
          b.planes = planes.data_ptr()
        elif isinstance(val, (torch.Tensor, np.ndarray)) and np.ndim(val) > 0:
          pl = _plane(val, di, shape3, dtype, device)
          planes = pl.unsqueeze(0).expand(hw, *pl.shape).contiguous()
          keep.append(planes)
          b.per_layer = 1
          b.planes = planes.data_ptr()
        else:
          b.value = float(val)
      elif kind == bc_types.BoundaryCondition.NEUMANN.value:
        if np.ndim(val) != 0:
          raise NotImplementedError('Only scalar Neumann values are supported.')
        b.kind = nat.SWC_BC_NEUMANN
        b.value = float(val)
      else:
        raise NotImplementedError(f'Unsupported BC type {sides[s][0]}.')
  return keep


class Solver:
  """One replica's grid, scheme and boundary conditions on the device."""

  def __init__(self, cfg, physics_models, shape: Sequence[int],
               dtype: torch.dtype = torch.float32,
               device: Optional[torch.device] = None, replica_id: int = 0,
               replicas: Optional[np.ndarray] = None,
               names: Optional[Sequence[str]] = None,
               interp_override: Optional[str] = None):
    nat.load()
    self.cfg = cfg
    self.pm = physics_models
    self.dtype = dtype
    self.device = device or torch.device('cuda', torch.cuda.current_device())
    names = list(names or cfg.conservative_variable_names)
    extra = [n for n in names if n not in types.BASE_CONSERVATIVE]
    missing = [n for n in types.BASE_CONSERVATIVE if n not in names]
    if missing:
      raise ValueError(f'Missing conservative variables {missing}.')
    if len(extra) > 3:
      raise NotImplementedError(
          f'{len(extra)} transported scalars {extra}; the fused CUDA path '
          'takes at most 3.')
    for n in extra:
      if not types.is_conservative_name(n):
        raise ValueError(f'Transported scalar "{n}" must be named rho_<name>.')
    # rho, rho_u, rho_v, rho_w, rho_e, then the scalars rho_phi.
    self.names = list(types.BASE_CONSERVATIVE) + extra
    self.ns = len(extra)
    hw = int(cfg.halo_width)
    nza, nxa, nya = (int(s) for s in shape)
    self.shape = (nza, nxa, nya)
    self.hw = hw
    self.nx, self.ny, self.nz = nxa - 2 * hw, nya - 2 * hw, nza - 2 * hw
    if min(self.nx, self.ny, self.nz) <= 0:
      raise ValueError(f'Field shape {shape} is too small for halo_width {hw}.')
    self.grid = nat.SwcGrid(self.nx, self.ny, self.nz, hw, nya, nya * nxa,
                            float(cfg.dx), float(cfg.dy), float(cfg.dz))
    sc = nat.SwcScheme()
    sc.dtype = nat.dtype_code(dtype)
    sc.interp = (_INTERP[interp_override] if interp_override
                 else interp_code(cfg))
    lim = getattr(cfg, 'muscl_limiter', 'mc')
    if lim not in _LIMITER:
      raise ValueError(f'Unknown MUSCL limiter "{lim}".')
    sc.limiter = _LIMITER[lim]
    sc.riemann = riemann_code(cfg)
    sc.diffusion = 1 if cfg.include_diffusion else 0
    sc.nscalars = self.ns
    sc.gravity_mask = physics_models.gravity_mask()
    sc.zseg = int(getattr(cfg, 'zseg', 0) or 0)
    sc.tile = int(getattr(cfg, 'tile', 0) or 0)
    sc.nu = physics_models.transport_model.nu
    sc.pr = physics_models.transport_model.pr
    for i, d in enumerate(types.DIMS):
      sc.g[i] = float(cfg.g[d])
    self._pe = [None, None, None]
    if utils.gravity_direction(cfg) != -1:
      reps = replicas if replicas is not None else np.array([[[0]]])
      mesh = utils.mesh_local(replica_id, reps, cfg)
      for i, d in enumerate(types.DIMS):
        coef = constant.G * float(cfg.g[d])
        if coef != 0.0:
          a = torch.as_tensor(coef * mesh[d].astype(np.float64), dtype=dtype)
          n_expect = {0: nxa, 1: nya, 2: nza}[i]
          if a.numel() != n_expect:
            raise ValueError(
                f'Mesh along {d} has {a.numel()} points with halos; the '
                f'fields have {n_expect}.')
          self._pe[i] = a.to(self.device).contiguous()
          sc.pe_axis[i] = self._pe[i].data_ptr()
    self.scheme = sc
    self.replica_id = int(replica_id)
    self.replicas = None if replicas is None else np.asarray(replicas)
    self._layout = None
    if self.replicas is not None and self.replicas.size > 1:
      from swirlc_b200 import halo_exchange as hx
      self._layout = hx.BlockLayout(self.replicas, hx.periodic_dims(cfg))
      glob = tuple(np.asarray(getattr(cfg, d)).shape[0] for d in ('z', 'x', 'y'))
      self._bc_cells = hx.localize_bc(cfg.bc.get(_CELL_AVG, {}), self.replicas,
                                      self.replica_id, hw, glob)
    else:
      self._bc_cells = cfg.bc.get(_CELL_AVG, {})
    self._build_bcs()
    self._build_ext()
    self._masked = None
    self._exchange = None
    if self._layout is not None:
      self._masked = hx.masked_bcs(self, self._layout, self.replica_id, nat)
    self._dt_cache: Dict[float, torch.Tensor] = {}

  # ------------------------------------------------------------------ BCs
  def _build_bcs(self):
    bc_all = self._bc_cells
    self._planes = []
    arr = (nat.SwcFieldBC * len(self.names))()
    for fi, name in enumerate(self.names):
      prim_name = types.conservative_to_primitive_name(name)
      if name in bc_all:
        spec, via = bc_all[name], 0
      elif prim_name in bc_all:
        spec, via = bc_all[prim_name], 1
      else:
        raise ValueError(
            'A "cells" boundary condition is required for all conservative'
            ' variables, either directly or through their respective'
            f' primitive. No boundary condition was found for {name} or'
            f' {prim_name}.')
      self._planes += fill_field_bc(arr[fi], spec, via, self.shape, self.hw,
                                    self.dtype, self.device, name)
    self.bcs = arr

  # ------------------------------------------------- face and flux BCs
  def _side_on_boundary(self, d: int, side: int) -> bool:
    """Whether this replica's side lies on the boundary of the whole grid
    (the only faces face/flux BCs act on, boundary.py:140-183, 434-461)."""
    if self.replicas is None or self.replicas.size == 1:
      return True
    c = np.argwhere(self.replicas == self.replica_id)[0]
    return c[d] == 0 if side == 0 else c[d] == self.replicas.shape[d] - 1

  def _override_value(self, o, val, d: int) -> None:
    if isinstance(val, (int, float, np.floating, np.integer)):
      o.value = float(val)
      o.plane = None
      return
    t = _plane(val, d, self.shape, self.dtype, self.device)
    self._planes.append(t)
    o.plane = t.data_ptr()

  def _build_ext(self) -> None:
    """SwcStageExt for the scalars and the cfg's face / flux BCs; use_ext
    tells whether the plain stage suffices."""
    e = nat.SwcStageExt()
    for d in range(3):
      for side in range(2):
        e.boundary[d][side] = int(self._side_on_boundary(d, side))
    prim_names = [types.conservative_to_primitive_name(n) if i else n
                  for i, n in enumerate(self.names)]
    faces = self.cfg.bc.get(_CELL_FACE) or {}
    for name, spec in faces.items():
      for d, dim in enumerate(types.DIMS):
        for side in range(2):
          kind, val = (spec.get(dim) or {}).get(side, (None, None))
          if kind is None:
            continue
          if bc_types.bc_value(kind) != bc_types.BoundaryCondition.DIRICHLET.value:
            raise ValueError(
                f'Unsupported interface (face or flux) BC type {kind}. Only'
                ' "DIRICHLET" or `None` is supported.')
          if name == types.RHO:
            raise NotImplementedError(
                'A density face boundary condition is not supported (the '
                'reference drops p and h from the face primitives after it).')
          if name in self.names:
            var, mode = self.names.index(name), nat.SWC_FACE_CONSERVATIVE
          elif name in prim_names:
            var, mode = prim_names.index(name), nat.SWC_FACE_PRIMITIVE
          else:
            raise ValueError(
                f'"{name}" is not a valid primitive or conservative variable'
                ' name for the face boundary condition update.')
          if not self._side_on_boundary(d, side):
            continue
          n = e.nface[d][side]
          o = e.face[d][side][n]
          o.var, o.mode = var, mode
          self._override_value(o, val, d)
          e.nface[d][side] = n + 1
    fluxes = self.cfg.bc.get(_CELL_FLUX) or {}
    codes = {bc_types.BoundaryFluxType.CONVECTIVE.value: nat.SWC_FLUX_CONVECTIVE,
             bc_types.BoundaryFluxType.DIFFUSIVE.value: nat.SWC_FLUX_DIFFUSIVE,
             bc_types.BoundaryFluxType.TOTAL.value: nat.SWC_FLUX_TOTAL}
    for ftype, per_var in fluxes.items():
      key = getattr(ftype, 'value', ftype)
      if key not in codes:
        raise ValueError(f'Unknown flux boundary type {ftype}.')
      for name, spec in per_var.items():
        if name not in self.names:
          raise ValueError(
              f'{name} cannot be specified by a flux boundary condition. Only'
              f' conservative variables {self.names} can be specified with a'
              ' flux boundary condition.')
        for d, dim in enumerate(types.DIMS):
          for side in range(2):
            kind, val = (spec.get(dim) or {}).get(side, (None, None))
            if kind is None or not self._side_on_boundary(d, side):
              continue
            if bc_types.bc_value(kind) != bc_types.BoundaryCondition.DIRICHLET.value:
              raise ValueError(
                  f'Unsupported interface (face or flux) BC type {kind}. Only'
                  ' "DIRICHLET" or `None` is supported.')
            n = e.nflux[d][side]
            o = e.flux[d][side][n]
            o.var, o.mode = self.names.index(name), codes[key]
            self._override_value(o, val, d)
            e.nflux[d][side] = n + 1
    if faces and self.cfg.include_diffusion:
      raise NotImplementedError(
          'Face boundary conditions are not supported with diffusion enabled'
          ' at this time.')
    has_overrides = any(e.nface[d][s] or e.nflux[d][s]
                        for d in range(3) for s in range(2))
    self.ext = e
    self.use_ext = bool(self.ns or has_overrides)

  # -------------------------------------------------------------- kernels
  def check_fields(self, fields: Sequence[torch.Tensor]) -> None:
    if len(fields) != len(self.names):
      raise ValueError(f'Expected {len(self.names)} conserved fields.')
    for f in fields:
      if (tuple(f.shape) != self.shape or f.dtype != self.dtype or
          not f.is_cuda or not f.is_contiguous()):
        raise ValueError(
            f'Field of shape {tuple(f.shape)} / {f.dtype} does not match the '
            f'solver ({self.shape}, {self.dtype}, contiguous CUDA).')

  def dt_tensor(self, dt: float) -> torch.Tensor:
    t = self._dt_cache.get(dt)
    if t is None:
      t = torch.tensor([float(dt)], dtype=torch.float64, device=self.device)
      self._dt_cache[dt] = t
    return t

  def fill_halos(self, fields: Sequence[torch.Tensor]) -> None:
    """In-place halo fill (boundary.update_conservative_cell_averages). With
    replicas > 1, halos on inner sides come from the neighbouring replicas
    over torch.distributed (rank = replica id), the others from the BCs."""
    if self._layout is not None:
      if self._exchange is None:
        from swirlc_b200 import halo_exchange as hx
        via = [self.bcs[i].via_primitive for i in range(len(self.bcs))]
        self._exchange = hx.DistExchange(
            self._layout, self.hw,
            lambda rid, fs, dim: self.fill_boundary_dim(fs, dim), via)
      self._exchange.fill([list(fields)], [self.replica_id])
      return
    ptrs = nat.ptr_array(fields)
    nat.check(nat.load().swc_halo_fill(
        ctypes.byref(self.grid), self.scheme.dtype, len(fields), ptrs,
        self.bcs, 0, nat.stream_ptr()), 'halo fill')

  def fill_boundary_dim(self, fields: Sequence[torch.Tensor], dim: int) -> None:
    """Halo fill along `dim` of the sides that take a boundary condition
    (not the sides shared with another replica)."""
    bcs = self._masked[dim] if self._masked is not None else None
    if bcs is None:
      from swirlc_b200 import halo_exchange as hx
      layout = hx.BlockLayout(np.zeros((1, 1, 1), np.int32), [False] * 3)
      self._masked = hx.masked_bcs(self, layout, 0, nat)
      bcs = self._masked[dim]
    nat.check(nat.load().swc_halo_fill(
        ctypes.byref(self.grid), self.scheme.dtype, len(fields),
        nat.ptr_array(fields), bcs, 0, nat.stream_ptr()), 'halo fill')

  def stage(self, uk, u0, uout, mode: int, c0: float = 0.0, c1: float = 0.0,
            dt: Optional[torch.Tensor] = None,
            dtmin_out: Optional[torch.Tensor] = None,
            helper: Optional[Dict[str, torch.Tensor]] = None) -> None:
    if self.use_ext or helper:
      e = self.ext
      if helper:
        e = nat.SwcStageExt.from_buffer_copy(self.ext)
        e.p_ref = self._helper_field(helper, 'p_ref').data_ptr()
        e.rho_ref = self._helper_field(helper, 'rho_ref').data_ptr()
      nat.check(nat.load().swc_rk_stage_ext(
          ctypes.byref(self.grid), ctypes.byref(self.scheme), ctypes.byref(e),
          nat.ptr_array(uk), nat.ptr_array(u0) if u0 is not None else None,
          nat.ptr_array(uout), mode, float(c0), float(c1),
          dt.data_ptr() if dt is not None else None,
          dtmin_out.data_ptr() if dtmin_out is not None else None,
          nat.stream_ptr()), 'rk stage')
      return
    nat.check(nat.load().swc_rk_stage(
        ctypes.byref(self.grid), ctypes.byref(self.scheme),
        nat.ptr_array(uk), nat.ptr_array(u0) if u0 is not None else None,
        nat.ptr_array(uout), mode, float(c0), float(c1),
        dt.data_ptr() if dt is not None else None,
        dtmin_out.data_ptr() if dtmin_out is not None else None,
        nat.stream_ptr()), 'rk stage')

  def stage_box(self, uk, u0, uout, mode: int, box: Sequence[int],
                c0: float = 0.0, c1: float = 0.0,
                dt: Optional[torch.Tensor] = None,
                dtmin_out: Optional[torch.Tensor] = None) -> None:
    """The fused stage on the interior sub-box box = (x0, x1, y0, y1, z0, z1)
    (interior cell indices, half-open) only. The same kernel runs on a grid
    whose origin is the box's first cell, with the whole array's strides:
    its stencils read the cells around the box, so a box at least
    halo_width cells away from every face reads no halo cell, and the boxes
    of a partition of the interior together give the whole stage bit for
    bit. Not for the extended stage (its face and flux BCs act on the
    grid's own faces)."""
    if self.use_ext:
      raise NotImplementedError('Sub-box stages need the plain fused stage.')
    x0, x1, y0, y1, z0, z1 = (int(v) for v in box)
    if not (0 <= x0 < x1 <= self.nx and 0 <= y0 < y1 <= self.ny and
            0 <= z0 < z1 <= self.nz):
      raise ValueError(f'Box {box} is not inside the {self.nx}x{self.ny}x'
                       f'{self.nz} interior.')
    g = nat.SwcGrid.from_buffer_copy(self.grid)
    g.nx, g.ny, g.nz = x1 - x0, y1 - y0, z1 - z0
    esz = torch.empty((), dtype=self.dtype).element_size()
    off = (z0 * self.grid.sz + x0 * self.grid.sx + y0) * esz
    sc = nat.SwcScheme.from_buffer_copy(self.scheme)
    for i, o in enumerate((x0, y0, z0)):
      if self.scheme.pe_axis[i]:
        sc.pe_axis[i] = self.scheme.pe_axis[i] + o * esz
    shift = lambda ts: nat.addr_array([t.data_ptr() + off for t in ts])
    nat.check(nat.load().swc_rk_stage(
        ctypes.byref(g), ctypes.byref(sc), shift(uk),
        shift(u0) if u0 is not None else None, shift(uout), mode, float(c0),
        float(c1), dt.data_ptr() if dt is not None else None,
        dtmin_out.data_ptr() if dtmin_out is not None else None,
        nat.stream_ptr()), 'rk stage (box)')

  def split_boxes(self, margin_xy: int = 16):
    """(inner, shell): the interior box whose stencils read no halo cell
    (halo_width planes from the z faces, `margin_xy` cells -- one 16-cell
    tile -- from the x and y faces) and the six boxes around it, or
    (None, []) when the grid is too small to split."""
    mz, m = self.hw, int(margin_xy)
    nx, ny, nz = self.nx, self.ny, self.nz
    if nx <= 2 * m or ny <= 2 * m or nz <= 2 * mz or m < self.hw:
      return None, []
    inner = (m, nx - m, m, ny - m, mz, nz - mz)
    shell = [(0, nx, 0, ny, 0, mz), (0, nx, 0, ny, nz - mz, nz),
             (0, m, 0, ny, mz, nz - mz), (nx - m, nx, 0, ny, mz, nz - mz),
             (m, nx - m, 0, m, mz, nz - mz),
             (m, nx - m, ny - m, ny, mz, nz - mz)]
    return inner, shell

  def _helper_field(self, helper, name) -> torch.Tensor:
    t = utils.as_tensor3d(helper[name])
    if (tuple(t.shape) != self.shape or t.dtype != self.dtype or
        not t.is_cuda or not t.is_contiguous()):
      raise ValueError(f'Helper variable {name} must be a contiguous CUDA '
                       f'tensor of shape {self.shape} and dtype {self.dtype}.')
    return t

  def cfl_reduce(self, fields, dtmin_out: torch.Tensor) -> None:
    nat.check(nat.load().swc_cfl_reduce(
        ctypes.byref(self.grid), ctypes.byref(self.scheme),
        nat.ptr_array(fields), dtmin_out.data_ptr(), nat.stream_ptr()),
        'cfl reduce')

  def new_fields(self, zero: bool = True) -> List[torch.Tensor]:
    alloc = torch.zeros if zero else torch.empty
    return [alloc(self.shape, dtype=self.dtype, device=self.device)
            for _ in range(len(self.names))]

  def rhs(self, fields: Sequence[torch.Tensor],
          helper: Optional[Dict[str, torch.Tensor]] = None) -> List[torch.Tensor]:
    """Functional RHS: copies, fills halos of the copy, returns dU/dt."""
    work = [f.clone() for f in fields]
    self.fill_halos(work)
    out = self.new_fields(zero=True)
    self.stage(work, None, out, nat.SWC_OUT_RHS, helper=helper)
    return out

  def rk3(self, fields: Sequence[torch.Tensor], dt: float,
          helper: Optional[Dict[str, torch.Tensor]] = None) -> List[torch.Tensor]:
    """Functional SSP-RK3 step (rk3.py:87-120) returning new fields."""
    dtt = self.dt_tensor(dt)
    u0 = [f.clone() for f in fields]
    self.fill_halos(u0)
    u1 = self.new_fields(zero=False)
    self.stage(u0, None, u1, nat.SWC_OUT_EULER, dt=dtt, helper=helper)
    self.fill_halos(u1)
    u2 = self.new_fields(zero=False)
    self.stage(u1, u0, u2, nat.SWC_OUT_CONVEX, 0.75, 0.25, dt=dtt,
               helper=helper)
    self.fill_halos(u2)
    self.stage(u2, u0, u1, nat.SWC_OUT_CONVEX, 1.0 / 3.0, 2.0 / 3.0, dt=dtt,
               helper=helper)
    self.fill_halos(u1)
    return u1

  def rk2(self, fields: Sequence[torch.Tensor], dt: float,
          helper: Optional[Dict[str, torch.Tensor]] = None) -> List[torch.Tensor]:
    """Functional RK2 step (rk2.py:63-86) returning new fields."""
    dtt = self.dt_tensor(dt)
    u0 = [f.clone() for f in fields]
    self.fill_halos(u0)
    u1 = self.new_fields(zero=False)
    self.stage(u0, None, u1, nat.SWC_OUT_EULER, dt=dtt, helper=helper)
    self.fill_halos(u1)
    u2 = self.new_fields(zero=False)
    self.stage(u1, u0, u2, nat.SWC_OUT_AVERAGE, 0.5, 0.0, dt=dtt,
               helper=helper)
    self.fill_halos(u2)
    return u2


class Stepper:
  """In-place time loop over a state with a device clock (no host syncs).

  Each step: [clock begin] -> fill(u) -> stage EULER u->w1 -> fill(w1) ->
  stage CONVEX (u, w1)->w2 -> fill(w2) -> stage CONVEX (u, w2)->u with the
  fused CFL reduction -> [clock end]. With `cfl` > 0 the step size is
  cfl * min(delta/(|u|+c)) computed on the device.
  """

  def __init__(self, solver: Solver, fields: Sequence[torch.Tensor],
               dt: float = 0.0, cfl: float = 0.0, t_end: float = 0.0,
               scheme: str = 'rk3',
               helper: Optional[Dict[str, torch.Tensor]] = None):
    solver.check_fields(fields)
    self.s = solver
    self.u = list(fields)
    self.w1 = solver.new_fields(zero=False)
    self.w2 = solver.new_fields(zero=False)
    self.scheme = scheme
    if scheme not in ('rk3', 'rk2'):
      raise NotImplementedError(f'"{scheme}" is not implemented as an '
                                '"time_integration_scheme".')
    # SwcClock: t, dt, dtmin, cfl, t_end, step (int64 bits in slot 5).
    self.clock = torch.zeros(6, dtype=torch.float64, device=solver.device)
    self.clock[1] = float(dt)
    self.clock[2] = 1e300
    self.clock[3] = float(cfl)
    self.clock[4] = float(t_end)
    self.cfl = float(cfl)
    self.helper = dict(helper) if helper else None
    if self.cfl > 0.0:
      solver.cfl_reduce(self.u, self.clock[2:3])
    self.graph: Optional[torch.cuda.CUDAGraph] = None

  @property
  def dt_ptr(self) -> torch.Tensor:
    return self.clock[1:2]

  def _launch_step(self):
    """One step through swc_rk_step (halo fills, fused stages, clock); the
    extended stage (scalars, helper states, face/flux BCs) is composed here
    from the same pieces."""
    if self.s.use_ext or self.helper:
      lib = nat.load()
      s, u, w1, w2 = self.s, self.u, self.w1, self.w2
      dt, dtmin = self.clock[1:2], self.clock[2:3]
      nat.check(lib.swc_clock_begin_step(self.clock.data_ptr(),
                                         nat.stream_ptr()))
      s.fill_halos(u)
      s.stage(u, None, w1, nat.SWC_OUT_EULER, dt=dt, helper=self.helper)
      s.fill_halos(w1)
      if self.scheme == 'rk3':
        s.stage(w1, u, w2, nat.SWC_OUT_CONVEX, 0.75, 0.25, dt=dt,
                helper=self.helper)
        s.fill_halos(w2)
        s.stage(w2, u, u, nat.SWC_OUT_CONVEX, 1.0 / 3.0, 2.0 / 3.0, dt=dt,
                dtmin_out=dtmin, helper=self.helper)
      else:
        s.stage(w1, u, u, nat.SWC_OUT_AVERAGE, 0.5, 0.0, dt=dt,
                dtmin_out=dtmin, helper=self.helper)
      nat.check(lib.swc_clock_end_step(self.clock.data_ptr(),
                                       nat.stream_ptr()))
      return
    work = self.w1 + self.w2
    nat.check(nat.load().swc_rk_step(
        ctypes.byref(self.s.grid), ctypes.byref(self.s.scheme), self.s.bcs,
        3 if self.scheme == 'rk3' else 2, nat.ptr_array(self.u),
        nat.ptr_array(work), self.clock.data_ptr(), nat.stream_ptr()),
        'rk step')

  def capture(self) -> None:
    """Captures one step in a CUDA graph (after one eager warm-up step)."""
    self.graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
      with torch.cuda.graph(self.graph, stream=side):
        self._launch_step()
    torch.cuda.current_stream().wait_stream(side)

  def step(self, n: int = 1, check: bool = False) -> None:
    """Advances n steps. With `check`, waits for them and raises
    FloatingPointError if the new state holds a non-finite rho, p or rho_e
    (or p/rho < 0), as flagged by the fused CFL reduction
    (swc_clock_status)."""
    for _ in range(n):
      if self.graph is not None:
        self.graph.replay()
      else:
        self._launch_step()
    if check:
      self.check()

  def check(self) -> None:
    """Raises FloatingPointError if the last step left a non-finite or
    unphysical state (waits for the current stream)."""
    nat.check(nat.load().swc_clock_status(self.clock.data_ptr(),
                                          nat.stream_ptr()), 'step')

  def time(self) -> float:
    return float(self.clock[0].item())

  def set_time(self, t: float, steps: int = 0) -> None:
    """Sets the clock's time and step count (a restarted run)."""
    self.clock[0] = float(t)
    self.clock[5:6].view(torch.int64).fill_(int(steps))

  def steps_done(self) -> int:
    return int(self.clock[5:6].view(torch.int64).item())
