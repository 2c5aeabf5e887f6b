"""GPU: a 1-D problem gives the same bits whichever axis it runs along.

The fused stage reconstructs x and y faces in the face form (two one-sided
reconstructions per face) and z faces in the cell-centred form (one per
cell, its upper-face value carried to the next plane), with the primitives
in two-lane pairs. All of these are written with the same explicitly rounded
operations, so a flow that varies along one axis only must come out of an
RK3 step bit for bit the same along x, y and z (with equal spacings), with
the momentum in the matching component and the other two exactly zero.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N, M, HW = 48, 8, 3
H = 1.0 / N


def _problem(axis, scheme, viscous):
  from swirlc_b200 import configs
  n = {'x': (N, M, M), 'y': (M, N, M), 'z': (M, M, N)}[axis]
  cfg = configs._base_cfg(n[0], n[1], n[2], n[0] * H, n[1] * H, n[2] * H, HW)
  cfg.update({'dx': H, 'dy': H, 'dz': H,
              'interpolation_scheme': scheme, 'numeric_flux_scheme': 'HLLC',
              'include_diffusion': viscous,
              'transport_parameters': {'nu': 2e-3, 'pr': 0.7},
              'time_integration_scheme': 'rk3',
              'bc': {'cell_averages': configs._periodic()}, 'dt': 1e-3})
  # Profile along the axis, halo cells included (periodic wrap).
  s = ((np.arange(N + 2 * HW) - HW + 0.5) % N) / N
  rho = 1.0 + 0.5 * (s > 0.5) + 0.1 * np.sin(2 * np.pi * s)
  p = 1.0 + 0.7 * (s < 0.25) + 0.05 * np.cos(6 * np.pi * s)
  un = 0.3 * np.sin(2 * np.pi * s) + 0.1
  e = p / (0.4 * rho) + 0.5 * un * un
  shape = tuple(k + 2 * HW for k in (n[2], n[0], n[1]))  # [z][x][y]
  where = {'x': (np.newaxis, slice(None), np.newaxis),
           'y': (np.newaxis, np.newaxis, slice(None)),
           'z': (slice(None), np.newaxis, np.newaxis)}[axis]

  def field(v):
    return (v[where] * np.ones(shape)).astype(np.float32)

  zero = np.zeros(shape, np.float32)
  mom = {'x': 'rho_u', 'y': 'rho_v', 'z': 'rho_w'}[axis]
  state = {'rho': field(rho), 'rho_u': zero, 'rho_v': zero, 'rho_w': zero,
           'rho_e': field(rho * e)}
  state[mom] = field(rho * un)
  return cfg, state, mom


def _line(f, axis):
  """The interior profile along `axis` (all transverse lines must agree)."""
  i = slice(HW, -HW)
  a = f[i, i, i]
  lines = {'x': a.permute(1, 0, 2).reshape(N, -1),
           'y': a.permute(2, 0, 1).reshape(N, -1),
           'z': a.reshape(N, -1)}[axis]
  assert torch.equal(lines, lines[:, :1].expand_as(lines)), axis
  return lines[:, 0]


@pytest.mark.parametrize('scheme,viscous', [('WENO_5', True),
                                            ('WENO_5', False),
                                            ('WENO_3', False),
                                            ('MUSCL', True)])
def test_one_dimensional_flow_is_axis_independent(scheme, viscous):
  from swirlc_b200 import engine
  from swirlc_b200.core import parameter
  from swirlc_b200.physics import physics_models
  names = ('rho', 'rho_u', 'rho_v', 'rho_w', 'rho_e')
  got = {}
  for axis in ('x', 'y', 'z'):
    user_cfg, state, mom = _problem(axis, scheme, viscous)
    cfg = parameter.SwirlCParameters(user_cfg)
    solver = engine.Solver(cfg, physics_models.PhysicsModels(cfg),
                           state['rho'].shape, torch.float32)
    f = [torch.tensor(state[k], device='cuda') for k in names]
    out = solver.rk3(f, 1e-3)
    torch.cuda.synchronize()
    res = dict(zip(names, out))
    got[axis] = {'rho': _line(res['rho'], axis),
                 'mom': _line(res[mom], axis),
                 'rho_e': _line(res['rho_e'], axis)}
    for k in ('rho_u', 'rho_v', 'rho_w'):
      if k != mom:
        assert not res[k][HW:-HW, HW:-HW, HW:-HW].any(), (axis, k)
  for axis in ('y', 'z'):
    for k in ('rho', 'mom', 'rho_e'):
      assert torch.equal(got[axis][k], got['x'][k]), (scheme, axis, k)
  # The step did something: the state moved away from its start.
  _, state, _ = _problem('x', scheme, viscous)
  start = torch.tensor(state['rho'][HW, HW:-HW, HW], device='cuda')
  assert not torch.equal(got['x']['rho'], start)
