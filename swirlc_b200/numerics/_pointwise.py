"""Shared launcher for the unit-level CUDA kernels (pointwise Riemann flux,
wave speeds, reconstruction and stencils) behind the reference's
function-level API."""

from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from swirlc_b200 import _native as nat
from swirlc_b200.common import types
from swirlc_b200.common import utils
from swirlc_b200.physics import constant

DIM_CODE = {'x': 0, 'y': 1, 'z': 2}


def dim_code(dim: str) -> int:
  if dim not in DIM_CODE:
    raise ValueError(
        f'"{dim}" is not a valid dimension. Available options are: "x", "y",'
        ' "z".')
  return DIM_CODE[dim]


def cuda3d(f, device=None) -> torch.Tensor:
  t = utils.as_tensor3d(f)
  if not t.is_cuda:
    t = t.to(device or torch.device('cuda', torch.cuda.current_device()))
  if t.dtype not in (torch.float32, torch.float64):
    t = t.to(torch.float32)
  return t.contiguous()


def array_grid(t: torch.Tensor) -> nat.SwcGrid:
  """SwcGrid covering a whole [nz, nx, ny] array (no halo)."""
  if t.dim() != 3:
    raise ValueError(f'Expected a 3-D field, got shape {tuple(t.shape)}.')
  nz, nx, ny = t.shape
  return nat.SwcGrid(nx, ny, nz, 0, ny, ny * nx, 1.0, 1.0, 1.0)


def potential_energy(cfg, shape, dtype, device, replica_id=0,
                     replicas=None) -> Optional[torch.Tensor]:
  """generic.py:282-319 on the cell-centre mesh, broadcast to `shape`, or
  None when cfg.g carries no gravity."""
  if cfg is None or utils.gravity_direction(cfg) == -1:
    return None
  reps = replicas if replicas is not None else np.array([[[0]]])
  mesh = utils.mesh_local(replica_id, reps, cfg)
  g = np.array([float(cfg.g[d]) for d in types.DIMS]) * constant.G
  x = mesh['x'][np.newaxis, :, np.newaxis].astype(np.float64)
  y = mesh['y'][np.newaxis, np.newaxis, :].astype(np.float64)
  z = mesh['z'][:, np.newaxis, np.newaxis].astype(np.float64)
  pe = (-g[0] * x - g[1] * y) - g[2] * z
  pe = np.broadcast_to(pe, tuple(shape))
  return torch.tensor(np.ascontiguousarray(pe), dtype=dtype, device=device)


def face_prims(prim: Dict, cons: Dict, scalars: Sequence[str],
               device) -> List[torch.Tensor]:
  """rho, u, v, w, e, p, h and scalars of one face side as flat tensors."""
  rho = cuda3d(prim[types.RHO], device)

  def get(name, cons_name=None):
    if name in prim:
      return cuda3d(prim[name], device)
    cn = cons_name or types.primitive_to_conservative_name(name)
    if cons and cn in cons:
      return cuda3d(cons[cn], device) / rho
    raise ValueError(f'Face state lacks "{name}".')

  out = [rho, get(types.U), get(types.V), get(types.W), get(types.E),
         cuda3d(prim[types.P], device), cuda3d(prim[types.H], device)]
  for s in scalars:
    out.append(get(types.conservative_to_primitive_name(s), s))
  dt = rho.dtype
  return [o.to(dt).reshape(-1).contiguous() for o in out]


def check_flux_fn(flux_fn, names: Sequence[str]) -> None:
  """Rejects a physical-flux function the fused kernel does not compute.

  The CUDA Riemann kernel evaluates the reference's physical flux
  (compressible_navier_stokes.py:338-427) itself. A `flux_fn` passed by the
  caller (hll.py:45, hllc.py:42) is accepted when it is None or computes
  that same flux; it is probed on a small float64 CPU state with
  h = e + p / rho, per conserved variable and dimension. Any other flux
  function raises NotImplementedError instead of being silently ignored.
  """
  if flux_fn is None:
    return
  from swirlc_b200.equations import compressible_navier_stokes as cns
  if flux_fn is cns._compute_physical_flux_1d:  # pylint: disable=protected-access
    return
  g = torch.Generator().manual_seed(0)
  r = lambda lo, hi: lo + (hi - lo) * torch.rand((2, 1, 1), generator=g,
                                                  dtype=torch.float64)
  prim = {types.RHO: r(0.5, 1.5), types.U: r(-1.0, 1.0),
          types.V: r(-1.0, 1.0), types.W: r(-1.0, 1.0), types.P: r(0.5, 2.0)}
  prim[types.E] = prim[types.P] / (0.4 * prim[types.RHO]) + r(0.0, 1.0)
  prim[types.H] = prim[types.E] + prim[types.P] / prim[types.RHO]
  cons = {types.RHO: prim[types.RHO]}
  for n in names:
    if n == types.RHO:
      continue
    pn = types.conservative_to_primitive_name(n)
    if pn not in prim:
      prim[pn] = r(0.0, 1.0)
    cons[n] = prim[types.RHO] * prim[pn]
  for dim in types.DIMS:
    vel = types.VELOCITY[types.DIMS.index(dim)]
    m = prim[types.RHO] * prim[vel]
    for n in names:
      pn = types.conservative_to_primitive_name(n)
      if pn == types.RHO:
        want = m
      elif pn == vel:
        want = m * prim[vel] + prim[types.P]
      elif pn == types.E:
        want = m * prim[types.H]
      else:
        want = m * prim[pn]
      try:
        got = torch.as_tensor(flux_fn(cons, prim, {}, dim, n),
                              dtype=torch.float64)
        ok = bool(torch.allclose(got, want, rtol=1e-12, atol=1e-12))
      except Exception as e:  # a flux function that cannot run on the probe
        raise NotImplementedError(
            'flux_fn must compute the physical convective flux '
            '(compressible_navier_stokes._compute_physical_flux_1d); the '
            f'probe call failed: {e!r}') from e
      if not ok:
        raise NotImplementedError(
            f'flux_fn differs from the physical convective flux for {n} '
            f'along {dim}; the CUDA Riemann kernel computes only that flux.')


def riemann_flux(riemann: int, conservative_neg, conservative_pos,
                 primitive_neg, primitive_pos, helper_var_neg, helper_var_pos,
                 dim: str, cfg, replica_id=0, replicas=None) -> Dict:
  d = dim_code(dim)
  names = list(getattr(cfg, 'conservative_variable_names',
                       types.BASE_CONSERVATIVE))
  scalars = [n for n in names if n not in types.BASE_CONSERVATIVE]
  ref = utils.as_tensor3d(primitive_neg[types.RHO])
  dev = ref.device if ref.is_cuda else torch.device(
      'cuda', torch.cuda.current_device())
  ql = face_prims(primitive_neg, conservative_neg, scalars, dev)
  qr = face_prims(primitive_pos, conservative_pos, scalars, dev)
  shape = tuple(utils.as_tensor3d(primitive_neg[types.RHO]).shape)
  dtype = ql[0].dtype
  n = ql[0].numel()
  pdl = pdr = None
  if helper_var_neg and 'p_dyn' in helper_var_neg:
    pdl = cuda3d(helper_var_neg['p_dyn'], dev).to(dtype).reshape(-1)
    pdr = cuda3d(helper_var_pos['p_dyn'], dev).to(dtype).reshape(-1)
  pe = potential_energy(cfg, shape, dtype, dev, replica_id, replicas)
  base = [torch.empty(n, dtype=dtype, device=dev) for _ in range(5)]
  extra = [torch.empty(n, dtype=dtype, device=dev) for _ in scalars]
  outs = base + extra
  nat.check(nat.load().swc_riemann_flux(
      n, nat.dtype_code(dtype), riemann, d, len(scalars), nat.ptr_array(ql),
      nat.ptr_array(qr), pdl.data_ptr() if pdl is not None else None,
      pdr.data_ptr() if pdr is not None else None,
      pe.reshape(-1).data_ptr() if pe is not None else None,
      nat.ptr_array(outs), nat.stream_ptr()), 'riemann flux')
  by_name = dict(zip(list(types.BASE_CONSERVATIVE) + scalars, outs))
  ref_in = primitive_neg[types.RHO]
  return {k: utils.like_input(by_name[k].reshape(shape), ref_in) for k in names}


def wave_speeds(primitive_neg, primitive_pos, dim: str, cfg, with_sm: bool,
                replica_id=0, replicas=None):
  d = dim_code(dim)
  ref = utils.as_tensor3d(primitive_neg[types.RHO])
  dev = ref.device if ref.is_cuda else torch.device(
      'cuda', torch.cuda.current_device())
  ql = face_prims(primitive_neg, None, (), dev)
  qr = face_prims(primitive_pos, None, (), dev)
  shape = tuple(ref.shape)
  dtype = ql[0].dtype
  n = ql[0].numel()
  pe = potential_energy(cfg, shape, dtype, dev, replica_id, replicas)
  s_l, s_r = (torch.empty(n, dtype=dtype, device=dev) for _ in range(2))
  s_m = torch.empty(n, dtype=dtype, device=dev) if with_sm else None
  nat.check(nat.load().swc_wave_speeds(
      n, nat.dtype_code(dtype), d, nat.ptr_array(ql), nat.ptr_array(qr),
      pe.reshape(-1).data_ptr() if pe is not None else None, s_l.data_ptr(),
      s_m.data_ptr() if s_m is not None else None, s_r.data_ptr(),
      nat.stream_ptr()), 'wave speeds')
  res = [s_l.reshape(shape)]
  if with_sm:
    res.append(s_m.reshape(shape))
  res.append(s_r.reshape(shape))
  return tuple(utils.like_input(r, primitive_neg[types.RHO]) for r in res)


def reconstruct(v, dim: str, interp: int, limiter: int = 0):
  t = cuda3d(v)
  neg, pos = torch.empty_like(t), torch.empty_like(t)
  grid = array_grid(t)
  nat.check(nat.load().swc_reconstruct(
      __import__('ctypes').byref(grid), nat.dtype_code(t.dtype), interp,
      limiter, dim_code(dim), t.data_ptr(), neg.data_ptr(), pos.data_ptr(),
      nat.stream_ptr()), 'reconstruct')
  return utils.like_input(neg, v), utils.like_input(pos, v)


def stencil(f, op: int, dim: str, h: float):
  t = cuda3d(f)
  out = torch.empty_like(t)
  grid = array_grid(t)
  nat.check(nat.load().swc_stencil(
      __import__('ctypes').byref(grid), nat.dtype_code(t.dtype), op,
      dim_code(dim), float(h), t.data_ptr(), out.data_ptr(),
      nat.stream_ptr()), 'stencil')
  return utils.like_input(out, f)


def viscous_terms(what: int, cell: Dict, cfg, rho_face=None, nu=None,
                  pr=None) -> List[torch.Tensor]:
  """swc_viscous_terms on whole 3-D arrays: cell values rho, u, v, w, p from
  `cell` (names the quantity does not read may be absent), spacings from
  cfg.dx/dy/dz, optional face densities [x, y, z]. Returns the output
  arrays in the C-ABI's order."""
  import ctypes
  names = (types.RHO, types.U, types.V, types.W, types.P)
  ref = next(cell[n] for n in names if n in cell)
  t0 = cuda3d(ref)
  dev, dtype = t0.device, t0.dtype
  q = [cuda3d(cell[n], dev).to(dtype).contiguous() if n in cell else None
       for n in names]
  rf = None
  if rho_face is not None:
    rf = [cuda3d(r, dev).to(dtype).contiguous() for r in rho_face]
  nz, nx, ny = t0.shape
  grid = nat.SwcGrid(nx, ny, nz, 0, ny, ny * nx, float(cfg.dx), float(cfg.dy),
                     float(cfg.dz))
  nout = {nat.SWC_VISC_FLUX: 15, nat.SWC_VISC_HEAT: 3}.get(what, 9)
  out = [torch.empty_like(t0) for _ in range(nout)]
  if nu is None:
    nu = cfg.transport_parameters['nu']
  if pr is None:
    pr = cfg.transport_parameters['pr']
  nat.check(nat.load().swc_viscous_terms(
      ctypes.byref(grid), nat.dtype_code(dtype), what, nat.ptr_array(q),
      nat.ptr_array(rf) if rf is not None else None, float(nu), float(pr),
      nat.ptr_array(out), nat.stream_ptr()), 'viscous terms')
  return out
