"""CPU: configuration, model selection and boundary-condition translation,
with the reference's error types (no GPU needed)."""

import numpy as np
import pytest
import torch

from swirlc_b200 import _native as nat
from swirlc_b200 import engine
from swirlc_b200.boundary import bc_types
from swirlc_b200.common import types, utils
from swirlc_b200.core import parameter
from swirlc_b200.numerics.riemann_solver import riemann_solver
from swirlc_b200.physics import physics_models

BC = bc_types.BoundaryCondition


def test_parameters_defaults_and_override():
  cfg = parameter.SwirlCParameters()
  assert cfg.halo_width == 3 and cfg.numeric_flux_scheme == 'HLL'
  assert cfg.conservative_variable_names == list(types.BASE_CONSERVATIVE)
  cfg2 = parameter.SwirlCParameters({'dt': 0.5, 'halo_width': 2})
  assert cfg2.dt == 0.5 and cfg2.halo_width == 2
  # Defaults are deep-copied (parameter.py:224-229).
  cfg2.bc['cell_averages'].clear()
  assert parameter.SwirlCParameters().bc['cell_averages']
  with pytest.raises(ValueError):
    parameter.SwirlCParameters({'kernel_op_type': 'bogus'})


def test_save_to_file(tmp_path):
  cfg = parameter.SwirlCParameters({'dt': 0.25})
  cfg.save_to_file(str(tmp_path / 'run'))
  assert (tmp_path / 'run_swirl_c_cfg.yml').exists()


def test_physics_models_selection_errors():
  with pytest.raises(NotImplementedError):
    physics_models.PhysicsModels(
        parameter.SwirlCParameters({'thermodynamics_model': 'x'}))
  with pytest.raises(NotImplementedError):
    physics_models.PhysicsModels(
        parameter.SwirlCParameters({'transport_model': 'x'}))
  with pytest.raises(NotImplementedError):
    physics_models.PhysicsModels(
        parameter.SwirlCParameters({'source_functions': ['x']}))
  with pytest.raises(ValueError):  # gravity without a direction
    physics_models.PhysicsModels(
        parameter.SwirlCParameters({'source_functions': ['gravity']}))
  pm = physics_models.PhysicsModels(parameter.SwirlCParameters(
      {'source_functions': ['gravity'], 'g': {'x': 0.0, 'y': 0.0, 'z': -1.0}}))
  assert pm.gravity_mask() == 4


def test_gravity_direction():
  cfg = parameter.SwirlCParameters({'g': {'x': 0.0, 'y': -1.0, 'z': 0.0}})
  assert utils.gravity_direction(cfg) == 1
  s = np.sqrt(0.5)
  cfg = parameter.SwirlCParameters({'g': {'x': s, 'y': 0.0, 'z': -s}})
  assert utils.gravity_direction(cfg) == 3
  assert utils.gravity_direction(parameter.SwirlCParameters()) == -1


def test_mesh_local_halo_rule():
  """utils.py:58-73: low halo coordinates are dx * [-hw..-1]."""
  cfg = parameter.SwirlCParameters()
  m = utils.mesh_local(0, np.array([[[0]]]), cfg)
  dx = cfg.x[1] - cfg.x[0]
  np.testing.assert_allclose(m['x'][:3], dx * np.array([-3, -2, -1]),
                             rtol=1e-6)
  np.testing.assert_allclose(m['x'][3:-3], cfg.x)


def test_scheme_selection_errors():
  with pytest.raises(ValueError):
    riemann_solver.select_numeric_flux_fn(
        parameter.SwirlCParameters({'numeric_flux_scheme': 'ROE'}))
  with pytest.raises(NotImplementedError):
    engine.interp_code(parameter.SwirlCParameters(
        {'interpolation_scheme': 'WENO_7'}))
  assert engine.interp_code(parameter.SwirlCParameters()) == nat.SWC_WENO5


def test_names():
  assert types.primitive_to_conservative_name('u') == 'rho_u'
  assert types.conservative_to_primitive_name('rho_e') == 'e'
  assert types.conservative_to_primitive_name('rho') == 'rho'
  with pytest.raises(ValueError):
    types.conservative_to_primitive_name('u')
  with pytest.raises(ValueError):
    types.primitive_to_conservative_name('')


def test_field_bc_translation():
  n = 16
  shape = (n, n, n)
  spec = {
      'x': {0: (BC.DIRICHLET, 8.0), 1: (BC.NEUMANN, 0.5)},
      'y': {0: (BC.PERIODIC,), 1: (BC.PERIODIC,)},
      'z': {0: (BC.DIRICHLET, [np.ones((n, n)) * k for k in (1, 2, 3)]),
            1: (BC.DIRICHLET, 0.0)},
  }
  fbc = nat.SwcFieldBC()
  keep = engine.fill_field_bc(fbc, spec, 0, shape, 3, torch.float32, 'cpu')
  assert fbc.side[0][0].kind == nat.SWC_BC_DIRICHLET
  assert fbc.side[0][0].value == 8.0 and fbc.side[0][0].per_layer == 0
  assert fbc.side[0][1].kind == nat.SWC_BC_NEUMANN
  assert fbc.side[1][0].kind == fbc.side[1][1].kind == nat.SWC_BC_PERIODIC
  assert fbc.side[2][0].per_layer == 1 and len(keep) == 1
  assert tuple(keep[0].shape) == (3, n, n)
  assert float(keep[0][2, 0, 0]) == 3.0
  with pytest.raises(NotImplementedError):
    engine.fill_field_bc(nat.SwcFieldBC(),
                         {'x': {0: (BC.REFLECTIVE, 0.0), 1: (BC.REFLECTIVE, 0)}},
                         0, shape, 3, torch.float32, 'cpu')
  with pytest.raises(ValueError):  # wrong number of layers
    engine.fill_field_bc(nat.SwcFieldBC(),
                         {'z': {0: (BC.DIRICHLET, [1.0, 2.0]),
                                1: (BC.DIRICHLET, 0.0)}},
                         0, shape, 3, torch.float32, 'cpu')


def test_product_never_imports_the_oracle():
  import os
  import re
  root = os.path.join(os.path.dirname(os.path.dirname(__file__)), 'swirlc_b200')
  for dirpath, _, files in os.walk(root):
    for f in files:
      if f.endswith('.py'):
        text = open(os.path.join(dirpath, f)).read()
        assert not re.search(r'^\s*(from|import)\s+oracle', text, re.M), f
