"""CPU oracle: a NumPy restatement of Swirl-C's compressible RHS + RK path.

TEST INFRASTRUCTURE ONLY. This module is the checker for the CUDA path: only
`tests/`, `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` may
import it. The product (`swirlc_b200`) never imports or calls it.

Every function restates the reference algorithm in plain NumPy, in the dtype
of its inputs (float32 or float64), following the operation order of the cited
reference lines (file:line, relative to the swirl_c project root). Arrays use
the reference layout `[nz, nx, ny]` (y contiguous) with halos included; 'x'
is axis 1, 'y' axis 2, 'z' axis 0.

Parity status:
  * Riemann solvers, physical flux, divergence, thermodynamics, transport,
    diffusion, gravity, halo fill, RK3/RK2 and the stencils are pinned by the
    reference's own known-answer tests (ported in tests/).
  * WENO5 (`weno(k=3)`), the prototype's MUSCL slope (`muscl(limiter=
    'minmod3')`), HLL, RK3 and the CFL rule are pinned to outputs of the
    reference's own NumPy prototype (demo/swirl_c_prototype.ipynb, cells 4,
    5, 11, 16), executed by tests/golden/make_prototype_fixtures.py; the two
    reconstructions agree bit for bit. The production reference calls its
    WENO and flux limiter in the un-vendored `swirl-lm` (pyproject.toml:32,
    bare git URL, no commit): the 'mc', 'van_leer' and 'minmod' limiters and
    WENO3 are restatements of the published schemes, parity unpinned.
"""

from __future__ import annotations

import copy
import math
from types import SimpleNamespace
from typing import Any, Dict, Optional, Sequence

import numpy as np

# physics/constant.py:17-41
G = 9.81
P_0 = 1.01325e5
GAMMA = 1.4
W_AIR = 0.029
R_U = 8.314
R = R_U / W_AIR
CV = R / (GAMMA - 1.0)
CP = CV + R
KAPPA = R / CP

# common/types.py:28
SMALL = np.finfo(np.float32).resolution

DIMS = ('x', 'y', 'z')
AXIS = {'x': 1, 'y': 2, 'z': 0}
RHO, U, V, W, E, P, H, T = 'rho', 'u', 'v', 'w', 'e', 'p', 'h', 't'
VELOCITY = (U, V, W)
RHO_U, RHO_V, RHO_W, RHO_E = 'rho_u', 'rho_v', 'rho_w', 'rho_e'
MOMENTUM = (RHO_U, RHO_V, RHO_W)
BASE_CONSERVATIVE = (RHO, RHO_U, RHO_V, RHO_W, RHO_E)
BASE_PRIMITIVES = (RHO, U, V, W, E)

PERIODIC, DIRICHLET, NEUMANN, REFLECTIVE = 0, 1, 2, 3
# Not a reference BC: the halo side is left as it is (a window cut out of a
# larger grid whose halo rows hold the neighbouring cells, as in the C-ABI's
# SWC_BC_NONE).
NONE = 4


def bc_kind(bc_type) -> int:
  """Maps an enum (reference bc_types.BoundaryCondition) or int to its value."""
  return int(getattr(bc_type, 'value', bc_type))


# ----------------------------------------------------------------------------
# Names (common/types.py:82-142)
# ----------------------------------------------------------------------------
def primitive_to_conservative_name(name: str) -> str:
  return RHO if name == RHO else 'rho_' + name


def conservative_to_primitive_name(name: str) -> str:
  if name == RHO:
    return RHO
  if name.startswith('rho_') and len(name) > 4:
    return name[4:]
  raise ValueError(f'Invalid conserved variable name: {name}.')


# ----------------------------------------------------------------------------
# Array helpers
# ----------------------------------------------------------------------------
def sh(v: np.ndarray, dim: str, k: int) -> np.ndarray:
  """Returns s with s[i] = v[i + k] along `dim` (wrapping at the array edge).

  Only interior results are ever compared, and every interior stencil stays
  inside the halo, so the wrap only touches undefined halo outputs.
  """
  return np.roll(v, -k, axis=AXIS[dim])


def divide_no_nan(x, y):
  """tf.math.divide_no_nan: 0 where y == 0."""
  x = np.asarray(x)
  y = np.asarray(y)
  safe = np.where(y == 0, np.ones_like(y), y)
  return np.where(y == 0, np.zeros_like(x * y), x / safe)


def reciprocal_no_nan(x):
  x = np.asarray(x)
  one = np.ones_like(x)
  return divide_no_nan(one, x)


def cfgget(cfg, key, default=None):
  if isinstance(cfg, dict):
    return cfg.get(key, default)
  return getattr(cfg, key, default)


# ----------------------------------------------------------------------------
# Mesh and gravity (common/utils.py:43-142; generic.py:282-319)
# ----------------------------------------------------------------------------
def mesh_local(cfg, core_idx=(0, 0, 0), dtype=np.float32) -> Dict[str, np.ndarray]:
  """common/utils.py:43-89 including the halo-coordinate quirk.

  The low halo coordinates are `dx * [-hw, ..., -1]` (utils.py:68), not
  `x[0] - dx * [hw, ..., 1]`.
  """
  hw = cfg.halo_width
  n_core = [cfg.cx, cfg.cy, cfg.cz]
  out = {}
  for i, dim in enumerate(DIMS):
    m = np.asarray(cfgget(cfg, dim), dtype=dtype)
    n_local = int(m.shape[0] / n_core[i])
    halo_lo = np.linspace(-hw, -1, hw).astype(dtype)
    halo_hi = np.linspace(1, hw, hw).astype(dtype)
    full = np.concatenate([(m[1] - m[0]) * halo_lo, m,
                           m[-1] + (m[-1] - m[-2]) * halo_hi])
    c = core_idx[i]
    idx = np.linspace(c * n_local, (c + 1) * n_local + 2 * hw - 1,
                      n_local + 2 * hw).astype(np.int32)
    out[dim] = full[idx]
  return out


def gravity_direction(cfg) -> int:
  """common/utils.py:114-142."""
  g = cfgget(cfg, 'g', {'x': 0.0, 'y': 0.0, 'z': 0.0})
  g_vec = np.array([g[d] for d in DIMS], dtype=float)
  if np.abs(np.linalg.norm(g_vec) - 1.0) >= SMALL:
    return -1
  for i in range(3):
    if np.abs(np.abs(g[DIMS[i]]) - 1.0) < SMALL:
      return i
  return 3


def potential_energy(cfg, shape, dtype, core_idx=(0, 0, 0)) -> np.ndarray:
  """generic.py:282-319: e_g = -g_vec . x on the cell-centre mesh."""
  if gravity_direction(cfg) == -1:
    return np.zeros(shape, dtype=dtype)
  mesh = mesh_local(cfg, core_idx, np.dtype(dtype).type)
  g = cfgget(cfg, 'g')
  g_vec = G * np.array([g[d] for d in DIMS], dtype=float)
  x = mesh['x'][np.newaxis, :, np.newaxis]
  y = mesh['y'][np.newaxis, np.newaxis, :]
  z = mesh['z'][:, np.newaxis, np.newaxis]
  t = np.dtype(dtype).type
  pe = (-t(g_vec[0]) * x - t(g_vec[1]) * y) - t(g_vec[2]) * z
  return np.broadcast_to(pe, shape).astype(dtype)


# ----------------------------------------------------------------------------
# Conversions and thermodynamics (common/utils.py:145-216; generic.py)
# ----------------------------------------------------------------------------
def conservative_to_primitive(cons: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
  """common/utils.py:145-183 (multiplies by tf.math.reciprocal(rho))."""
  rho = cons[RHO]
  inv_rho = (np.ones_like(rho) / rho)
  prim = {RHO: rho}
  for key, val in cons.items():
    if key == RHO:
      continue
    if key.startswith('rho_') and len(key) > 4:
      prim[key[4:]] = inv_rho * val
  return prim


def primitive_to_conservative(prim: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
  """common/utils.py:186-216."""
  out = {}
  for key, val in prim.items():
    if key == RHO:
      out[RHO] = prim[RHO]
    else:
      out['rho_' + key] = prim[RHO] * val
  return out


def internal_energy(states, pe):
  """generic.py:357-389."""
  u, v, w = states[U], states[V], states[W]
  return states[E] - 0.5 * (u**2 + v**2 + w**2) - pe


def pressure(states, pe):
  """generic.py:27-57."""
  return (GAMMA - 1.0) * states[RHO] * internal_energy(states, pe)


def total_enthalpy(states, pe):
  """generic.py:59-87."""
  return states[E] + pressure(states, pe) / states[RHO]


def sensible_enthalpy(states, pe):
  """generic.py:391-423."""
  u, v, w = states[U], states[V], states[W]
  return states[H] - 0.5 * (u**2 + v**2 + w**2) - pe


def sound_speed(states, pe=0.0, opt='e'):
  """generic.py:90-158."""
  if opt == 'e':
    return np.sqrt(GAMMA * (GAMMA - 1.0) * internal_energy(states, pe))
  if opt == 'h':
    return np.sqrt((GAMMA - 1.0) * sensible_enthalpy(states, pe))
  if opt == 'p_rho':
    return np.sqrt(GAMMA * states[P] / states[RHO])
  raise ValueError(f'"{opt}" is not a valid option for sound speed.')


def temperature_eos(states):
  """generic.py:223-228."""
  return states[P] / (states[RHO] * R)


# ----------------------------------------------------------------------------
# Stencils (numerics/gradient.py:21-94; numerics/interpolation.py:21-53)
# ----------------------------------------------------------------------------
def forward_1(f, h, dim):
  return (sh(f, dim, 1) - f) / h


def backward_1(f, h, dim):
  return (f - sh(f, dim, -1)) / h


def central_2(f, h, dim):
  return (sh(f, dim, 1) - sh(f, dim, -1)) / (2.0 * h)


def linear_interpolation(f, dim):
  """Face i-1/2 value 0.5 * (f[i-1] + f[i])."""
  return 0.5 * (sh(f, dim, -1) + f)


# ----------------------------------------------------------------------------
# Face reconstruction (swirl_lm weno / flux_limiter; restated from the
# prototype demo/swirl_c_prototype.ipynb `weno5` and `muscl`, cell 4)
# ----------------------------------------------------------------------------
_WENO_C = {
    3: {-1: (11.0 / 6.0, -7.0 / 6.0, 1.0 / 3.0),
        0: (1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0),
        1: (-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0),
        2: (1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0)},
    2: {-1: (1.5, -0.5),
        0: (0.5, 0.5),
        1: (-0.5, 1.5)},
}
_WENO_D = {3: (0.3, 0.6, 0.1), 2: (2.0 / 3.0, 1.0 / 3.0)}
WENO_EPS = 1e-6


def _weno_betas(v, dim, k):
  vm2, vm1, v0, vp1, vp2 = (sh(v, dim, -2), sh(v, dim, -1), v, sh(v, dim, 1),
                            sh(v, dim, 2))
  if k == 3:
    # prototype beta_0/1/2 on (v_i, v_i+1, v_i+2), (v_i-1, v_i, v_i+1),
    # (v_i-2, v_i-1, v_i).
    b0 = (13.0 / 12.0 * (v0 - 2.0 * vp1 + vp2)**2
          + 0.25 * (3.0 * v0 - 4.0 * vp1 + vp2)**2)
    b1 = (13.0 / 12.0 * (vm1 - 2.0 * v0 + vp1)**2 + 0.25 * (vm1 - vp1)**2)
    b2 = (13.0 / 12.0 * (vm2 - 2.0 * vm1 + v0)**2
          + 0.25 * (vm2 - 4.0 * vm1 + 3.0 * v0)**2)
    return (b0, b1, b2)
  # WENO3-JS smoothness of the two 2-point stencils.
  return ((vp1 - v0)**2, (v0 - vm1)**2)


def _weno_cell(v, dim, k):
  """Per cell i: (right-face i+1/2 value, left-face i-1/2 value).

  Mirrors the prototype: vr_neg[r] = sum_j c[r][j] v[i-r+j],
  vr_pos[r] = sum_j c[r-1][j] v[i-r+j]; alpha = d / (eps + beta)**2.
  """
  c = _WENO_C[k]
  d = _WENO_D[k]
  beta = _weno_betas(v, dim, k)
  zero = np.zeros_like(v)
  vr_neg, vr_pos = [], []
  for r in range(k):
    bn = zero.copy()
    bp = zero.copy()
    for j in range(k):
      s = sh(v, dim, -r + j)
      bn = bn + c[r][j] * s
      bp = bp + c[r - 1][j] * s
    vr_neg.append(bn)
    vr_pos.append(bp)
  a_neg, a_pos = [], []
  s_neg = zero.copy()
  s_pos = zero.copy()
  for r in range(k):
    a_neg.append(d[r] / (WENO_EPS + beta[r])**2)
    a_pos.append(d[k - 1 - r] / (WENO_EPS + beta[r])**2)
    s_neg = s_neg + a_neg[r]
    s_pos = s_pos + a_pos[r]
  out_neg = zero.copy()
  out_pos = zero.copy()
  for r in range(k):
    out_neg = out_neg + (a_neg[r] / s_neg) * vr_neg[r]
    out_pos = out_pos + (a_pos[r] / s_pos) * vr_pos[r]
  return out_neg, out_pos


def weno(v, dim, k=3):
  """Returns (neg, pos) at face i-1/2 (compressible_navier_stokes.py:581-615).

  neg[i]: reconstruction from the left cell i-1 (stencil i-1-k+1..i-1+k-1);
  pos[i]: reconstruction from the right cell i.
  """
  right_face, left_face = _weno_cell(v, dim, k)
  return sh(right_face, dim, -1), left_face


MUSCL_LIMITERS = ('van_leer', 'mc', 'minmod', 'minmod3')


def _limiter(r, kind):
  if kind == 'van_leer':
    # From |r| >= 2^54 (2^25 in float32) 1 + |r| rounds to |r| and the
    # formula gives exactly 2 (r > 0) or 0 (r < 0). Those values are taken
    # directly there, which also covers ratios where r + |r| overflows or r
    # is infinite (float64 keeps subnormals, so dm / dp overflows when dp is
    # one), for which the formula gives inf or NaN. The CUDA limiter does
    # the same.
    a = np.abs(r)
    big = 2.0 ** 54 if r.dtype == np.float64 else 2.0 ** 25
    with np.errstate(invalid='ignore', over='ignore'):
      phi = (r + a) / (1.0 + a)
    return np.where(a >= big, np.where(r > 0, 2.0, 0.0), phi).astype(
        phi.dtype, copy=False)
  if kind == 'mc':
    return np.maximum(0.0, np.minimum(np.minimum(2.0 * r, 0.5 * (1.0 + r)), 2.0))
  if kind == 'minmod':
    return np.maximum(0.0, np.minimum(r, 1.0))
  raise ValueError(f'Unknown limiter {kind}.')


def _minmod3_slope(v, dim):
  """The prototype's MUSCL slope (swirl_c_prototype.ipynb `muscl`, cell 4).

  minmod of the central difference (v[c+1]-v[c-1])/(2*2) (its `central2`
  with h = 2), the forward difference and the backward difference (h = 1):
  s = mean of the three signs, the slope is s * min |.| where |s| == 1, else 0.
  """
  grads = ((sh(v, dim, 1) - sh(v, dim, -1)) / (2.0 * 2.0),
           (sh(v, dim, 1) - v) / 1.0,
           (v - sh(v, dim, -1)) / 1.0)
  s = (np.sign(grads[0]) + np.sign(grads[1]) + np.sign(grads[2])) / 3
  a_min = np.minimum(np.minimum(np.abs(grads[0]), np.abs(grads[1])),
                     np.abs(grads[2]))
  return np.where(np.abs(s) == 1, s * a_min, np.zeros_like(a_min)).astype(
      v.dtype, copy=False)


def muscl(v, dim, limiter='mc'):
  """Slope-limited MUSCL reconstruction at face i-1/2.

  For cell c: dp = v[c+1]-v[c], dm = v[c]-v[c-1], r = divide_no_nan(dm, dp),
  slope = phi(r) * dp ('minmod3': the prototype's three-slope minmod).
  neg[i] = v[i-1] + 0.5 slope[i-1]; pos[i] = v[i] - 0.5 slope[i].
  """
  if limiter == 'minmod3':
    slope = _minmod3_slope(v, dim)
  else:
    dp = sh(v, dim, 1) - v
    dm = v - sh(v, dim, -1)
    r = divide_no_nan(dm, dp)
    slope = _limiter(r, limiter) * dp
  right_face = v + 0.5 * slope
  left_face = v - 0.5 * slope
  return sh(right_face, dim, -1), left_face


def node_interp(v, dim):
  """Identity face values (the reference tests' `weno` mock, cns_test.py:55-60)."""
  del dim
  return v, v


def face_interp_fn(cfg):
  scheme = cfgget(cfg, 'interpolation_scheme')
  if scheme == 'WENO_3':
    return lambda v, d: weno(v, d, 2)
  if scheme == 'WENO_5':
    return lambda v, d: weno(v, d, 3)
  if scheme == 'MUSCL':
    lim = cfgget(cfg, 'muscl_limiter', 'mc')
    return lambda v, d: muscl(v, d, lim)
  if scheme == 'NODE':
    return node_interp
  raise NotImplementedError(f'"{scheme}" is not implemented as an '
                            '"interpolation_scheme".')


# ----------------------------------------------------------------------------
# Physical flux and Riemann solvers
# ----------------------------------------------------------------------------
def physical_flux_1d(cons, prim, helper, dim, var_name):
  """compressible_navier_stokes.py:338-427."""
  p_updated = helper.get('p_dyn', prim[P])
  var = conservative_to_primitive_name(var_name)
  aligned_vel = VELOCITY[DIMS.index(dim)]
  aligned_mom = primitive_to_conservative_name(aligned_vel)
  if var == aligned_vel:
    return cons[aligned_mom] * prim[aligned_vel] + p_updated
  if var == E:
    return cons[aligned_mom] * (prim[E] + prim[P] / prim[RHO])
  if var == RHO:
    return cons[aligned_mom]
  return cons[aligned_mom] * prim[var]


def hll_wave_speeds(prim_neg, prim_pos, dim, pe):
  """hll.py:178-283."""
  aligned = VELOCITY[DIMS.index(dim)]
  c_neg = sound_speed(prim_neg, opt='p_rho')
  c_pos = sound_speed(prim_pos, opt='p_rho')
  rn = np.sqrt(prim_neg[RHO])
  rp = np.sqrt(prim_pos[RHO])
  inv = reciprocal_no_nan(rn + rp)
  roe = {}
  for name in list(VELOCITY) + [H]:
    roe[name] = (rn * prim_neg[name] + rp * prim_pos[name]) * inv
  roe_c = sound_speed(roe, pe, opt='h')
  s_l = np.minimum(prim_neg[aligned] - c_neg, roe[aligned] - roe_c)
  s_r = np.maximum(prim_pos[aligned] + c_pos, roe[aligned] + roe_c)
  return s_l, s_r


def hll_flux(cons_neg, cons_pos, prim_neg, prim_pos, help_neg, help_pos, dim,
             var_names, pe, flux_fn=physical_flux_1d):
  """hll.py:36-175."""
  s_l, s_r = hll_wave_speeds(prim_neg, prim_pos, dim, pe)
  ds = s_r - s_l
  t1 = divide_no_nan(np.minimum(s_r, 0.0) - np.minimum(s_l, 0.0), ds)
  t2 = np.ones_like(t1) - t1
  t3 = divide_no_nan(s_r * np.abs(s_l) - s_l * np.abs(s_r), 2.0 * ds)
  out = {}
  for name in var_names:
    fn = flux_fn(cons_neg, prim_neg, help_neg, dim, name)
    fp = flux_fn(cons_pos, prim_pos, help_pos, dim, name)
    out[name] = t1 * fp + t2 * fn - t3 * (cons_pos[name] - cons_neg[name])
  return out


def hllc_wave_speeds(prim_neg, prim_pos, dim, pe):
  """hllc.py:260-347."""
  aligned = VELOCITY[DIMS.index(dim)]
  v_l, v_r = prim_neg[aligned], prim_pos[aligned]
  rho_l, rho_r = prim_neg[RHO], prim_pos[RHO]
  p_l, p_r = prim_neg[P], prim_pos[P]
  s_l, s_r = hll_wave_speeds(prim_neg, prim_pos, dim, pe)
  s_m = divide_no_nan(
      p_r - p_l + rho_l * v_l * (s_l - v_l) - rho_r * v_r * (s_r - v_r),
      rho_l * (s_l - v_l) - rho_r * (s_r - v_r))
  s_m = np.where(np.abs(s_m) < 1e-6, np.zeros_like(s_m), s_m)
  return s_l, s_m, s_r


def hllc_flux(cons_neg, cons_pos, prim_neg, prim_pos, help_neg, help_pos, dim,
              var_names, pe, flux_fn=physical_flux_1d):
  """hllc.py:33-257."""

  def updated(prim, helper):
    out = dict(prim)
    if 'p_dyn' in helper:
      out[P] = helper['p_dyn']
    return out

  pn = updated(prim_neg, help_neg)
  pp = updated(prim_pos, help_pos)
  s_l, s_m, s_r = hllc_wave_speeds(pn, pp, dim, pe)
  aligned = VELOCITY[DIMS.index(dim)]

  def star(prim_k, s_k, f_k, name):
    var = conservative_to_primitive_name(name)
    rho_k, v_k = prim_k[RHO], prim_k[aligned]
    if var == RHO:
      return f_k + rho_k * (s_m - v_k) * divide_no_nan(s_k, s_k - s_m)
    if var == E:
      return (f_k + rho_k * divide_no_nan(s_k, s_k - s_m) * (s_m - v_k)
              * (prim_k[E] + prim_k[P] / rho_k + (s_k - v_k) * s_m))
    if var == aligned:
      return f_k + rho_k * s_k * (divide_no_nan(s_k - v_k, s_k - s_m) * s_m - v_k)
    return (f_k + rho_k * (s_m - v_k) * prim_k[var]
            * divide_no_nan(s_k, s_k - s_m))

  out = {}
  for name in var_names:
    f_l = flux_fn(cons_neg, prim_neg, help_neg, dim, name)
    f_r = flux_fn(cons_pos, prim_pos, help_pos, dim, name)
    f_ml = star(pn, s_l, f_l, name)
    f_mr = star(pp, s_r, f_r, name)
    out[name] = np.where(
        s_l >= 0.0, f_l,
        np.where((s_l <= 0.0) & (s_m >= 0.0), f_ml,
                 np.where((s_m <= 0.0) & (s_r >= 0.0), f_mr, f_r)))
  return out


# ----------------------------------------------------------------------------
# Diffusion (physics/fluid.py:31-111; physics/diffusion.py:33-109;
# compressible_navier_stokes.py:618-707)
# ----------------------------------------------------------------------------
def strain_rate(prim, delta):
  """fluid.py:31-111; element [i][j] lives on the j face."""

  def grad(f, gd, fd):
    h = delta[gd]
    if gd == fd:
      return backward_1(f, h, gd)
    return linear_interpolation(central_2(f, h, gd), fd)

  u, v, w = prim[U], prim[V], prim[W]
  dudx = {fd: grad(u, 'x', fd) for fd in DIMS}
  dvdy = {fd: grad(v, 'y', fd) for fd in DIMS}
  dwdz = {fd: grad(w, 'z', fd) for fd in DIMS}
  div = {fd: dudx[fd] + dvdy[fd] + dwdz[fd] for fd in DIMS}
  sd = lambda g, d: g - 1.0 / 3.0 * d
  so = lambda a, b: 0.5 * (a + b)
  return [
      [sd(dudx['x'], div['x']), so(grad(u, 'y', 'y'), grad(v, 'x', 'y')),
       so(grad(u, 'z', 'z'), grad(w, 'x', 'z'))],
      [so(grad(v, 'x', 'x'), grad(u, 'y', 'x')), sd(dvdy['y'], div['y']),
       so(grad(v, 'z', 'z'), grad(w, 'y', 'z'))],
      [so(grad(w, 'x', 'x'), grad(u, 'z', 'x')),
       so(grad(w, 'y', 'y'), grad(v, 'z', 'y')), sd(dwdz['z'], div['z'])],
  ]


def shear_stress(prim, prim_f, delta, nu):
  """diffusion.py:33-67: tau_ij = 2 rho_j nu s_ij on face j."""
  s = strain_rate(prim, delta)
  rho = [prim_f[d][RHO] for d in DIMS]
  return [[2.0 * rho[j] * nu * s[i][j] for j in range(3)] for i in range(3)]


def heat_flux(prim, delta, nu, pr):
  """diffusion.py:76-109 with transport/simple.py:81-107."""
  t = temperature_eos(prim)
  mu = nu * prim[RHO]
  kappa = (1.0 / pr) * (CP * np.ones_like(prim[RHO])) * mu
  out = {}
  for d in DIMS:
    kf = linear_interpolation(kappa, d)
    out[d] = -kf * backward_1(t, delta[d], d)
  return out


def diffusive_flux(prim, cfg, var_names):
  """compressible_navier_stokes.py:618-707."""
  tp = cfgget(cfg, 'transport_parameters')
  nu, pr = tp['nu'], tp['pr']
  delta = {'x': cfg.dx, 'y': cfg.dy, 'z': cfg.dz}
  prim_f = {d: {k: linear_interpolation(prim[k], d)
                for k in list(VELOCITY) + [RHO]} for d in DIMS}
  tau = shear_stress(prim, prim_f, delta, nu)
  q = heat_flux(prim, delta, nu, pr)
  flux = {d: {k: np.zeros_like(prim[RHO]) for k in var_names} for d in DIMS}
  for j, d in enumerate(DIMS):
    for i in range(3):
      flux[d][MOMENTUM[i]] = -tau[i][j]
  for j, d in enumerate(DIMS):
    vel = [prim_f[d][k] for k in VELOCITY]
    tb = [tau[i][j] for i in range(3)]
    flux[d][RHO_E] = -(vel[0] * tb[0] + vel[1] * tb[1] + vel[2] * tb[2])
  for d in DIMS:
    flux[d][RHO_E] = q[d] + flux[d][RHO_E]
  return flux


# ----------------------------------------------------------------------------
# Halo fill (boundary/boundary.py:34-86, 464-539; swirl_lm halo exchange
# semantics pinned by boundary/boundary_test.py:60-343)
# ----------------------------------------------------------------------------
def _set_plane(v, axis, idx, val):
  sl = [slice(None)] * 3
  sl[axis] = idx
  sl = tuple(sl)
  if np.isscalar(val) or np.ndim(val) == 0:
    v[sl] = val
  else:
    v[sl] = np.asarray(val).reshape(v[sl].shape)


def _get_plane(v, axis, idx):
  sl = [slice(None)] * 3
  sl[axis] = idx
  return v[tuple(sl)]


def exchange_halos(u, bc_dim: Dict[str, Any], hw: int) -> np.ndarray:
  """Single-replica halo fill, dims in order x, y, z (boundary.py:34-86).

  PERIODIC wraps; DIRICHLET writes a scalar into every layer or layer l of a
  per-layer list (index 0 outermost on the low side, innermost on the high
  side); NEUMANN extrapolates halo = neighbour -/+ value layer by layer.
  """
  u = np.array(u, copy=True)
  for dim in DIMS:
    if dim not in bc_dim or not bc_dim[dim]:
      continue
    ax = AXIS[dim]
    n = u.shape[ax]
    sides = bc_dim[dim]
    if bc_kind(sides[0][0]) == PERIODIC or bc_kind(sides[1][0]) == PERIODIC:
      for l in range(hw):
        _set_plane(u, ax, l, _get_plane(u, ax, n - 2 * hw + l).copy())
        _set_plane(u, ax, n - hw + l, _get_plane(u, ax, hw + l).copy())
      continue
    for side in (0, 1):
      kind = bc_kind(sides[side][0])
      if kind == NONE:
        continue
      val = sides[side][1]
      if kind == DIRICHLET:
        for l in range(hw):
          lv = val[l] if isinstance(val, (list, tuple)) else val
          idx = l if side == 0 else n - hw + l
          _set_plane(u, ax, idx, np.asarray(lv, dtype=u.dtype) if not np.isscalar(lv) else lv)
      elif kind == NEUMANN:
        for l in range(hw):
          if side == 0:
            src = _get_plane(u, ax, hw - l)
            _set_plane(u, ax, hw - 1 - l, src - u.dtype.type(val))
          else:
            src = _get_plane(u, ax, n - hw - 1 + l)
            _set_plane(u, ax, n - hw + l, src + u.dtype.type(val))
      else:
        raise NotImplementedError(f'Unsupported BC type {kind}.')
  return u


def update_conservative_cell_averages(cons, cfg):
  """boundary.py:464-539 (single replica)."""
  bc = cfgget(cfg, 'bc')['cell_averages']
  hw = cfg.halo_width
  out = dict(cons)
  for name in list(out.keys()):
    if name in bc:
      out[name] = exchange_halos(out[name], bc[name], hw)
    elif conservative_to_primitive_name(name) in bc:
      prim = divide_no_nan(out[name], out[RHO])
      prim = exchange_halos(prim, bc[conservative_to_primitive_name(name)], hw)
      out[name] = out[RHO] * prim
    else:
      raise ValueError('A "cells" boundary condition is required for all '
                       f'conservative variables. None for {name}.')
  return out


# ----------------------------------------------------------------------------
# RHS (compressible_navier_stokes.py:68-268)
# ----------------------------------------------------------------------------
def _interface_bc(bc_by_var, dim, side):
  """boundary.py:186-236 (_get_bc_dict_along_dim): DIRICHLET or None."""
  out = {}
  for name, spec in bc_by_var.items():
    kind, val = spec[dim][side]
    if kind is None:
      continue
    if bc_kind(kind) != DIRICHLET:
      raise AssertionError(f'Unsupported interface (face or flux) BC type {kind}.')
    out[name] = val
  return out


def _plane_value(val, like):
  if np.isscalar(val) or np.ndim(val) == 0:
    return like.dtype.type(val)
  return np.asarray(val, dtype=like.dtype)


def update_faces(c_neg, c_pos, p_neg, p_pos, cfg):
  """boundary.py:340-461 with _face_boundary_update_1d (:239-337), one
  replica: face values on the planes between halo and interior; as in the
  reference, the other member of the (conservative, primitive) pair is then
  recomputed over the whole array. A density face BC is applied first and
  rebuilds the face primitives from the conservative values (:279-293), which
  drops p and h, as the reference does."""
  bcf = (cfgget(cfg, 'bc') or {}).get('cell_faces')
  if not bcf:
    return
  hw = cfg.halo_width
  for d in DIMS:
    ax = AXIS[d]
    for side in (0, 1):
      bc1 = _interface_bc(bcf, d, side)
      if not bc1:
        continue
      for cd, pd in ((c_neg, p_neg), (c_pos, p_pos)):
        cons = cd[d]
        n = cons[RHO].shape[ax] - 2 * hw
        idx = hw if side == 0 else hw + n
        if RHO in bc1:
          _set_plane(cons[RHO], ax, idx, _plane_value(bc1[RHO], cons[RHO]))
          pd[d] = conservative_to_primitive(cons)
        prim = pd[d]
        for name, val in bc1.items():
          if name == RHO:
            continue
          if name in cons:
            pname = conservative_to_primitive_name(name)
            _set_plane(cons[name], ax, idx, _plane_value(val, cons[name]))
            prim[pname] = divide_no_nan(cons[name], cons[RHO])
          else:
            cname = 'rho_' + name
            _set_plane(prim[name], ax, idx, _plane_value(val, prim[name]))
            cons[cname] = cons[RHO] * prim[name]


def update_fluxes(flux, cfg, flux_type: str):
  """boundary.py:89-183, one replica: the flux across the boundary faces
  (indices hw and hw + n along the dim) set for the given flux type."""
  bcx = (cfgget(cfg, 'bc') or {}).get('intercell_fluxes')
  if not bcx or flux_type not in bcx:
    return flux
  hw = cfg.halo_width
  for d in DIMS:
    ax = AXIS[d]
    for side in (0, 1):
      for name, val in _interface_bc(bcx[flux_type], d, side).items():
        f = flux[d][name]
        n = f.shape[ax] - 2 * hw
        _set_plane(f, ax, hw if side == 0 else hw + n, _plane_value(val, f))
  return flux


def rhs(cons: Dict[str, np.ndarray], cfg, helper: Optional[Dict] = None,
        interp_fn=None, apply_bc=True, pe=None, conv_flux_fn=None,
        diff_flux_fn=None, grad_fn=None, source_fn=None
        ) -> Dict[str, np.ndarray]:
  """compressible_navier_stokes.py:68-268.

  The keyword hooks stand where the reference's own tests patch it:
  `interp_fn` for swirl_lm's weno, `apply_bc=False` for
  update_conservative_cell_averages, `conv_flux_fn(c_neg, c_pos, p_neg,
  p_pos)` for _intercell_convective_flux (returns {dim: {var: flux}}),
  `diff_flux_fn(prim)` for _intercell_diffusive_flux, `grad_fn(f, h, dim)`
  for gradient.forward_1 in the divergence, and `source_fn(cons)` for
  physics_models.source_function (added to the gravity source).
  """
  helper = dict(helper or {})
  if apply_bc:
    cons = update_conservative_cell_averages(dict(cons), cfg)
  names = list(cons.keys())
  dtype = cons[RHO].dtype
  if pe is None:
    pe = potential_energy(cfg, cons[RHO].shape, dtype)
  prim = conservative_to_primitive(cons)
  prim[P] = pressure(prim, pe)
  prim[H] = prim[E] + prim[P] / prim[RHO]
  face_vars = []
  if 'p_ref' in helper and 'rho_ref' in helper:
    zero_bc = {d: {0: (DIRICHLET, 0.0), 1: (DIRICHLET, 0.0)} for d in DIMS}
    helper['p_dyn'] = exchange_halos(prim[P] - helper['p_ref'], zero_bc,
                                     cfg.halo_width)
    helper['d_rho'] = exchange_halos(prim[RHO] - helper['rho_ref'], zero_bc,
                                     cfg.halo_width)
    face_vars.append('p_dyn')
  interp = interp_fn or face_interp_fn(cfg)
  prim_names = cfgget(cfg, 'primitive_variable_names',
                      [conservative_to_primitive_name(n) for n in names])
  fi = {k: {d: interp(v, d) for d in DIMS} for k, v in prim.items()}
  hi = {k: {d: interp(helper[k], d) for d in DIMS} for k in face_vars}
  p_neg = {d: {k: fi[k][d][0] for k in fi} for d in DIMS}
  p_pos = {d: {k: fi[k][d][1] for k in fi} for d in DIMS}
  h_neg = {d: {k: hi[k][d][0] for k in hi} for d in DIMS}
  h_pos = {d: {k: hi[k][d][1] for k in hi} for d in DIMS}
  c_neg = {d: primitive_to_conservative({k: p_neg[d][k] for k in prim_names})
           for d in DIMS}
  c_pos = {d: primitive_to_conservative({k: p_pos[d][k] for k in prim_names})
           for d in DIMS}
  update_faces(c_neg, c_pos, p_neg, p_pos, cfg)
  scheme = cfgget(cfg, 'numeric_flux_scheme')
  if scheme == 'HLL':
    ffn = hll_flux
  elif scheme == 'HLLC':
    ffn = hllc_flux
  else:
    raise ValueError(f'"{scheme}" is not implemented as a "numeric_flux_scheme".')
  if conv_flux_fn is not None:
    flux = conv_flux_fn(c_neg, c_pos, p_neg, p_pos)
  else:
    flux = {d: ffn(c_neg[d], c_pos[d], p_neg[d], p_pos[d], h_neg[d],
                   h_pos[d], d, names, pe) for d in DIMS}
  flux = update_fluxes(flux, cfg, 'convective')
  if cfgget(cfg, 'include_diffusion', False):
    dflux = (diff_flux_fn(prim) if diff_flux_fn is not None
             else diffusive_flux(prim, cfg, names))
    fd = update_fluxes(dflux, cfg, 'diffusive')
    for d in DIMS:
      for k in names:
        flux[d][k] = flux[d][k] + fd[d][k]
  flux = update_fluxes(flux, cfg, 'total')
  source = {k: np.zeros_like(v) for k, v in cons.items()}
  src_fns = cfgget(cfg, 'source_functions') or []
  if 'gravity' in src_fns:
    gdir = gravity_direction(cfg)
    if gdir == -1:
      raise ValueError('Gravity direction must be specified if the gravity '
                       'source function is to be used.')
    g = cfgget(cfg, 'g')
    d_rho = helper.get('d_rho', cons[RHO])
    mask = MOMENTUM if gdir == 3 else (MOMENTUM[gdir],)
    for i, d in enumerate(DIMS):
      if MOMENTUM[i] in mask:
        source[MOMENTUM[i]] = source[MOMENTUM[i]] + d_rho * G * g[d]
  if source_fn is not None:
    extra = source_fn(cons)
    for k in names:
      source[k] = source[k] + extra[k]
  delta = {'x': cfg.dx, 'y': cfg.dy, 'z': cfg.dz}
  grad = grad_fn or forward_1
  for k in names:
    for d in DIMS:
      source[k] = source[k] - grad(flux[d][k], delta[d], d)
  return source


# ----------------------------------------------------------------------------
# Time integration (rk3.py:24-122; rk2.py:63-86)
# ----------------------------------------------------------------------------
RK3_C11, RK3_C21 = 0.75, 1.0 / 3.0
RK3_C12, RK3_C22 = 1.0 - RK3_C11, 1.0 - RK3_C21


def rk3(state0, dt, rhs_fn):
  l = rhs_fn(state0)
  s1 = {k: v + l[k] * dt for k, v in state0.items()}
  l = rhs_fn(s1)
  s2 = {k: v * RK3_C11 + (s1[k] + l[k] * dt) * RK3_C12 for k, v in state0.items()}
  l = rhs_fn(s2)
  return {k: v * RK3_C21 + (s2[k] + l[k] * dt) * RK3_C22 for k, v in state0.items()}


def rk2(state0, dt, rhs_fn):
  l = rhs_fn(state0)
  s1 = {k: v + dt * l[k] for k, v in state0.items()}
  l = rhs_fn(s1)
  s2 = {k: v + dt * l[k] for k, v in s1.items()}
  return {k: 0.5 * (v + s2[k]) for k, v in state0.items()}


def cfl_dt_min(cons, cfg, pe=None):
  """min over interior cells and dims of delta_d / (|u_d| + c).

  CFL rule of the prototype's diagnostic (swirl_c_prototype.ipynb `solve`,
  cell 16), with c = sqrt(gamma p / rho) and p from generic.py:27-57.
  """
  hw = cfg.halo_width
  if pe is None:
    pe = potential_energy(cfg, cons[RHO].shape, cons[RHO].dtype)
  prim = conservative_to_primitive(cons)
  p = pressure(prim, pe)
  # Interior cells only: halo layers may hold values no fill has set.
  sl = (slice(hw, -hw or None),) * 3
  c = np.sqrt(GAMMA * p[sl] / prim[RHO][sl])
  dts = []
  for d, vel in zip(DIMS, VELOCITY):
    delta = {'x': cfg.dx, 'y': cfg.dy, 'z': cfg.dz}[d]
    dts.append(np.min(delta / (np.abs(prim[vel][sl]) + c)))
  return float(min(dts))


# ----------------------------------------------------------------------------
# Config helper
# ----------------------------------------------------------------------------
def periodic_bc(names=BASE_CONSERVATIVE):
  return {'cell_averages': {
      n: {d: {0: (PERIODIC,), 1: (PERIODIC,)} for d in DIMS} for n in names}}


def make_cfg(**kw) -> SimpleNamespace:
  """A SwirlCParameters-like namespace with the reference defaults (parameter.py:44-131)."""
  xx = np.linspace(0.0, 1.0, 11, dtype=np.float32)
  xx = xx[:-1] + 0.5 * np.diff(xx)[0]
  base = dict(
      cx=1, cy=1, cz=1, halo_width=3, nx=10, ny=10, nz=10,
      x=xx, y=xx, z=xx, dx=float(np.diff(xx)[0]), dy=float(np.diff(xx)[0]),
      dz=float(np.diff(xx)[0]), g={'x': 0.0, 'y': 0.0, 'z': 0.0}, dt=1e-3,
      interpolation_scheme='WENO_5', numeric_flux_scheme='HLL',
      include_diffusion=False, time_integration_scheme='rk3',
      source_functions=None, transport_parameters={'nu': 1.0e-4, 'pr': 0.7},
      conservative_variable_names=list(BASE_CONSERVATIVE),
      primitive_variable_names=list(BASE_PRIMITIVES), bc=periodic_bc())
  base.update(copy.deepcopy(kw))
  return SimpleNamespace(**base)
