"""Golden vectors from the reference's own runnable NumPy prototype.

The reference's production path calls WENO and the MUSCL flux limiter in the
un-vendored `swirl-lm`, and its RHS tests mock them. The only in-tree,
runnable statement of that arithmetic is the NumPy prototype notebook
demo/swirl_c_prototype.ipynb. This script executes the notebook's own
function definitions (cells 4, 5, 8, 9 and 11: `weno5`, `muscl`, `rk3`,
`primitive_variables`, `sound_speed`, `convective_flux`, `hll`) and the CFL
expression of its `solve` loop (cell 16), on seeded inputs, and writes the
results in the production convention of this repository's tests:

  * arrays in the reference layout [nz, nx, ny] ('x' axis 1, 'y' axis 2,
    'z' axis 0); the prototype stores [nx, ny, nz];
  * face index i holds face i-1/2 (the prototype stores face i+1/2 at i), neg
    from the left cell's stencil, pos from the right cell's.

Only definitions are executed (no plotting cell, no simulation cell). It needs
NumPy only:

  python tests/golden/make_prototype_fixtures.py /path/to/swirl_c \
      > tests/golden/prototype_vectors.json
"""

import enum
import json
import os
import sys

import numpy as np

# Notebook cells holding the definitions used here (0-based cell index).
_CELLS = (4, 5, 8, 9, 11)
_SOLVE_CELL = 16


def load_prototype(root: str) -> dict:
  path = os.path.join(root, 'demo', 'swirl_c_prototype.ipynb')
  with open(path) as f:
    nb = json.load(f)
  ns = {'np': np, 'enum': enum}
  for i in _CELLS:
    exec(compile(''.join(nb['cells'][i]['source']), f'cell{i}', 'exec'), ns)
  # rk3 applies the notebook's update_boundary (cell 2, BC machinery) after
  # each stage; the fixtures step unbounded arrays, so it is the identity.
  ns['update_boundary'] = lambda states, params: states
  src = ''.join(nb['cells'][_SOLVE_CELL]['source'])
  return ns, src


def cfl_numbers(ns: dict, solve_src: str, states, params):
  """The per-axis CFL numbers exactly as `solve` (cell 16) prints them.

  The three `cfl_*` assignment lines are taken from the cell's source text
  and evaluated on the given states.
  """
  lines = [l.strip() for l in solve_src.splitlines()
           if l.strip().startswith(('var = primitive_variables', 'c = sound_speed',
                                    'cfl_x =', 'cfl_y =', 'cfl_z ='))]
  assert len(lines) == 5, lines
  local = dict(ns)
  local.update(states=states, params=params)
  for l in lines:
    exec(l, local)
  return [float(local['cfl_x']), float(local['cfl_y']), float(local['cfl_z'])]


# Prototype axis of each dim in [nx, ny, nz]; ours is [nz, nx, ny].
_PAXIS = {'x': 0, 'y': 1, 'z': 2}


def enc(a):
  """Nested lists; float32 values as the shortest decimal that reads back
  to the same float32."""
  a = np.asarray(a)
  if a.dtype == np.float32:
    return np.vectorize(lambda x: float(np.format_float_positional(
        x, unique=True, trim='-')), otypes=[object])(a).tolist() if a.ndim else \
        float(np.format_float_positional(a, unique=True, trim='-'))
  return a.tolist()


def to_ref_layout(a):
  return enc(np.ascontiguousarray(np.transpose(a, (2, 0, 1))))


def shift_to_i_minus_half(a, dim):
  """Prototype face i+1/2 at index i -> face i-1/2 at index i."""
  return np.roll(a, 1, axis=_PAXIS[dim])


def fields(kind: str, shape, dim, rng):
  n = shape[_PAXIS[dim]]
  s = np.arange(n, dtype=np.float64)
  bshape = [1, 1, 1]
  bshape[_PAXIS[dim]] = n
  s = s.reshape(bshape)
  noise = rng.standard_normal(shape)
  if kind == 'smooth':
    v = 1.0 + 0.5 * np.sin(2 * np.pi * s / n + 0.3) + 0.01 * noise
  elif kind == 'discontinuous':
    v = np.where(s < n // 2, 1.0, 0.125) + 0.02 * np.cos(s) + 0.001 * noise
  elif kind == 'near_flat':
    v = 2.5 + 1e-7 * noise
  elif kind == 'rough':
    v = rng.standard_normal(shape)
  else:
    raise ValueError(kind)
  return np.broadcast_to(v, shape).copy()


def valid_ranges(dim_len, scheme):
  """Index ranges [lo, hi) (production convention) where neg / pos are set."""
  if scheme == 'weno5':
    return (3, dim_len - 1), (2, dim_len - 2)
  # muscl: neg[i] = right face of cell i-1 (needs i-2..i), pos[i] = left face
  # of cell i (needs i-1..i+1).
  return (2, dim_len), (1, dim_len - 1)


def recon_cases(ns, rng):
  out = []
  for scheme in ('weno5', 'muscl'):
    for dt in ('float64', 'float32'):
      for dim in ('x', 'y', 'z'):
        for kind in ('smooth', 'discontinuous', 'near_flat', 'rough'):
          shape = [2, 2, 2]
          shape[_PAXIS[dim]] = 14
          v = fields(kind, tuple(shape), dim, rng).astype(dt)
          neg, pos = ns[scheme](v, dim)
          assert neg.dtype == np.dtype(dt) and pos.dtype == np.dtype(dt)
          neg = shift_to_i_minus_half(neg, dim)
          pos = shift_to_i_minus_half(pos, dim)
          n = shape[_PAXIS[dim]]
          (nlo, nhi), (plo, phi) = valid_ranges(n, scheme)
          out.append({
              'scheme': scheme, 'dtype': dt, 'dim': dim, 'kind': kind,
              'v': to_ref_layout(v),
              'neg': to_ref_layout(neg),
              'pos': to_ref_layout(pos),
              'neg_range': [nlo, nhi], 'pos_range': [plo, phi]})
  return out


def random_cons(rng, shape, dt, gravity_z=None):
  rho = 0.5 + rng.random(shape)
  u = rng.uniform(-1.0, 1.0, shape)
  v = rng.uniform(-1.0, 1.0, shape)
  w = rng.uniform(-1.0, 1.0, shape)
  p = 0.5 + 2.0 * rng.random(shape)
  e = p / (0.4 * rho) + 0.5 * (u * u + v * v + w * w)
  if gravity_z is not None:
    e = e + 9.81 * gravity_z
  c = {'rho': rho, 'rhou': rho * u, 'rhov': rho * v, 'rhow': rho * w,
       'rhoe': rho * e}
  return {k: a.astype(dt) for k, a in c.items()}


_CONS_MAP = {'rho': 'rho', 'rhou': 'rho_u', 'rhov': 'rho_v', 'rhow': 'rho_w',
             'rhoe': 'rho_e'}


def hll_cases(ns, rng):
  out = []
  ns['params'] = {}  # hll reads the notebook's global params (no gravity)
  for dt in ('float64', 'float32'):
    for d, dim in enumerate(('x', 'y', 'z')):
      shape = (24,)
      neg = random_cons(rng, shape, dt)
      pos = random_cons(rng, shape, dt)
      # A few equal and mirror states (u~ = 0, U_R - U_L = 0 cases).
      for k in neg:
        pos[k][:4] = neg[k][:4]
      fneg = ns['convective_flux'](neg, neg, neg, {})
      fpos = ns['convective_flux'](pos, pos, pos, {})
      f_neg = {k: v[d] for k, v in fneg.items()}
      f_pos = {k: v[d] for k, v in fpos.items()}
      flux = ns['hll'](neg, pos, f_neg, f_pos, d)
      out.append({
          'dtype': dt, 'dim': dim,
          'cons_neg': {_CONS_MAP[k]: enc(a) for k, a in neg.items()},
          'cons_pos': {_CONS_MAP[k]: enc(a) for k, a in pos.items()},
          'flux': {_CONS_MAP[k]: enc(a) for k, a in flux.items()}})
  return out


def rk3_cases(ns, rng):
  out = []
  for dt in ('float64', 'float32'):
    s0 = {'rho': rng.random(16).astype(dt), 'rhou': rng.random(16).astype(dt)}
    a = rng.uniform(-2.0, 2.0, 16).astype(dt)
    b = rng.uniform(-1.0, 1.0, 16).astype(dt)

    def rhs_fn(states, helper_vars, params, a=a, b=b):
      del helper_vars, params
      return {k: a * v + b for k, v in states.items()}

    step = 0.05
    res = ns['rk3'](rhs_fn, s0, {}, {'dt': step})
    out.append({'dtype': dt, 'dt': step, 'a': enc(a), 'b': enc(b),
                'state0': {_CONS_MAP[k]: enc(v) for k, v in s0.items()},
                'state1': {_CONS_MAP[k]: enc(v) for k, v in res.items()}})
  return out


def cfl_cases(ns, solve_src, rng):
  out = []
  for dt in ('float64', 'float32'):
    for grav in (False, True):
      shape = (8, 5, 4)  # prototype [nx, ny, nz], interior cells only
      dx, dy, dz = 0.1, 0.07, 0.13
      x = (np.arange(shape[0]) + 0.5) * dx
      y = (np.arange(shape[1]) + 0.5) * dy
      z = (np.arange(shape[2]) + 0.5) * dz
      zz = np.broadcast_to(z[np.newaxis, np.newaxis, :], shape) if grav else None
      cons = random_cons(rng, shape, dt, gravity_z=zz)
      params = {'dx': dx, 'dy': dy, 'dz': dz, 'dt': 1e-3}
      if grav:
        params.update({'x': x.astype(dt), 'y': y.astype(dt), 'z': z.astype(dt),
                       'g': {'x': 0.0, 'y': 0.0, 'z': -1.0}})
      cfl = cfl_numbers(ns, solve_src, cons, params)
      out.append({'dtype': dt, 'gravity_z': grav, 'dx': dx, 'dy': dy,
                  'dz': dz, 'dt': params['dt'], 'x': x.tolist(),
                  'y': y.tolist(), 'z': z.tolist(),
                  'cons': {_CONS_MAP[k]: to_ref_layout(a)
                           for k, a in cons.items()},
                  'cfl_xyz': cfl})
  return out


def main(root: str) -> dict:
  ns, solve_src = load_prototype(root)
  rng = np.random.default_rng(20241)
  return {
      'source': 'demo/swirl_c_prototype.ipynb (cells 4, 5, 8, 9, 11, 16)',
      'layout': '[nz, nx, ny]; face index i holds face i-1/2',
      'recon': recon_cases(ns, rng),
      'hll': hll_cases(ns, rng),
      'rk3': rk3_cases(ns, rng),
      'cfl': cfl_cases(ns, solve_src, rng),
  }


if __name__ == '__main__':
  json.dump(main(sys.argv[1]), sys.stdout)
  sys.stdout.write('\n')
