"""Shared test helpers: seeded states, configs, comparisons."""

import copy

import numpy as np

from oracle import swirlc_oracle as orc

DIMS = ('x', 'y', 'z')


def to_3d(f, dim, size):
  """Tiles a 1-D profile along `dim` into [nz, nx, ny] (the reference's
  common/testing_utils.py:23-62 layout)."""
  f = np.asarray(f)
  if dim == 'x':
    return np.tile(f[np.newaxis, :, np.newaxis], (size[0], 1, size[2]))
  if dim == 'y':
    return np.tile(f[np.newaxis, np.newaxis, :], (size[0], size[1], 1))
  return np.tile(f[:, np.newaxis, np.newaxis], (1, size[1], size[2]))


def rel_l2(a, b, hw=0):
  a = np.asarray(a, dtype=np.float64)
  b = np.asarray(b, dtype=np.float64)
  if hw:
    a = a[hw:-hw, hw:-hw, hw:-hw]
    b = b[hw:-hw, hw:-hw, hw:-hw]
  den = np.linalg.norm(b)
  return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def random_state(shape, seed=0, dtype=np.float32, gravity_pe=None):
  """A smooth-ish random compressible state with positive rho and p."""
  rng = np.random.default_rng(seed)
  nz, nx, ny = shape
  z, x, y = np.meshgrid(np.linspace(0, 2 * np.pi, nz),
                        np.linspace(0, 2 * np.pi, nx),
                        np.linspace(0, 2 * np.pi, ny), indexing='ij')
  rho = 1.0 + 0.2 * np.sin(x + 0.3) * np.cos(y) + 0.05 * rng.random(shape)
  u = 0.3 * np.sin(y + z) + 0.05 * rng.standard_normal(shape)
  v = 0.2 * np.cos(x - z) + 0.05 * rng.standard_normal(shape)
  w = 0.25 * np.sin(x + y) + 0.05 * rng.standard_normal(shape)
  p = 1.0 + 0.1 * np.cos(x) * np.sin(z) + 0.02 * rng.random(shape)
  pe = 0.0 if gravity_pe is None else gravity_pe
  e = p / (0.4 * rho) + 0.5 * (u * u + v * v + w * w) + pe
  cons = {'rho': rho, 'rho_u': rho * u, 'rho_v': rho * v, 'rho_w': rho * w,
          'rho_e': rho * e}
  return {k: np.asarray(v, dtype=dtype) for k, v in cons.items()}


def periodic_bc(names=orc.BASE_CONSERVATIVE):
  return orc.periodic_bc(names)
