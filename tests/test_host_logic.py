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


def _same(a, b):
  if isinstance(a, dict):
    return a.keys() == b.keys() and all(_same(a[k], b[k]) for k in a)
  if isinstance(a, (list, tuple)):
    return (type(a) is type(b) and len(a) == len(b)
            and all(_same(x, y) for x, y in zip(a, b)))
  if isinstance(a, np.ndarray):
    return (isinstance(b, np.ndarray) and a.dtype == b.dtype
            and np.array_equal(a, b))
  return type(a) is type(b) and a == b


@pytest.mark.parametrize('case', ['default', 'bubble', 'kh'])
def test_config_yaml_round_trip(tmp_path, case):
  """save_to_file -> load_from_file rebuilds the same dictionary: NumPy
  mesh arrays and scalars (dtype kept), BC enum tuples, Dirichlet planes."""
  from swirlc_b200 import configs
  user = {'default': lambda: None,
          'bubble': lambda: configs.buoyant_bubble(nx=8, ny=8, nz=6)[0],
          'kh': lambda: configs.kelvin_helmholtz(n=8)[0]}[case]()
  cfg = parameter.SwirlCParameters(user)
  prefix = str(tmp_path / 'sub' / case)
  cfg.save_to_file(prefix)
  back = parameter.SwirlCParameters.load_from_file(prefix)
  assert _same(cfg._simulation_cfg, back._simulation_cfg)
  back2 = parameter.SwirlCParameters.load_from_file(
      prefix + '_swirl_c_cfg.yml')
  assert _same(cfg._simulation_cfg, back2._simulation_cfg)


def test_config_yaml_loader_rejects_other_python_objects(tmp_path):
  import yaml
  for text in ('x: !!python/object/apply:os.getcwd []\n',
               'x: !!python/name:os.system \'\'\n',
               'x: !!python/object:collections.OrderedDict {}\n'):
    p = tmp_path / 'bad_swirl_c_cfg.yml'
    p.write_text(text)
    with pytest.raises(yaml.YAMLError):
      parameter.SwirlCParameters.load_from_file(str(p))


@pytest.mark.parametrize('dtype', [torch.float32, torch.float64])
def test_state_files_round_trip(tmp_path, dtype):
  from swirlc_b200.core import state_io
  g = torch.Generator().manual_seed(0)
  state = {k: torch.rand((7, 9, 11), generator=g, dtype=dtype)
           for k in types.BASE_CONSERVATIVE}
  prefix = str(tmp_path / 'a' / 'run')
  state_io.save_state(prefix, state, 40, coordinate=(1, 0, 2), t=0.125)
  assert (tmp_path / 'a' / 'run-field-rho_e-xyz-1-0-2-step-40.npy').exists()
  back, t = state_io.load_state(prefix, types.BASE_CONSERVATIVE, 40,
                                coordinate=(1, 0, 2))
  assert t == 0.125
  for k in state:
    assert back[k].dtype == dtype and torch.equal(back[k], state[k])
  back64, _ = state_io.load_state(prefix, ['rho'], 40, (1, 0, 2),
                                  dtype=torch.float64)
  assert back64['rho'].dtype == torch.float64
  state_io.save_state(prefix, {'rho': state['rho']}, 41)
  assert state_io.load_state(prefix, ['rho'], 41)[1] is None
  with pytest.raises(FileNotFoundError):
    state_io.load_state(prefix, ['rho'], 39, (1, 0, 2))
  with pytest.raises(KeyError):
    state_io.save_state(prefix, state, 42, names=['rho_y'])
  state_io.save_state(prefix, {'rho': state['rho'],
                               'rho_u': state['rho_u'][:, :, :5]}, 43)
  with pytest.raises(ValueError):
    state_io.load_state(prefix, ['rho', 'rho_u'], 43)
  assert not list((tmp_path / 'a').glob('*.tmp*'))


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


def test_riemann_flux_fn_is_checked_not_dropped():
  """hll/hllc_convective_flux accept None, the reference's physical flux and
  any function that computes it (the reference tests pass their own), and
  raise for another flux instead of silently using the built-in one."""
  from swirlc_b200.equations import compressible_navier_stokes as cns
  from swirlc_b200.numerics import _pointwise
  names = list(types.BASE_CONSERVATIVE) + ['rho_y']
  _pointwise.check_flux_fn(None, names)
  _pointwise.check_flux_fn(cns._compute_physical_flux_1d, names)

  def from_enthalpy(cons, prim, helper, dim, name):
    del cons, helper
    var = types.conservative_to_primitive_name(name)
    vel = types.VELOCITY[types.DIMS.index(dim)]
    m = prim['rho'] * prim[vel]
    if var == 'rho':
      return m
    if var == vel:
      return m * prim[vel] + prim['p']
    if var == 'e':
      return m * prim['h']
    return m * prim[var]

  _pointwise.check_flux_fn(from_enthalpy, names)
  with pytest.raises(NotImplementedError):
    _pointwise.check_flux_fn(
        lambda c, p, h, d, n: 2.0 * from_enthalpy(c, p, h, d, n), names)
  with pytest.raises(NotImplementedError):
    _pointwise.check_flux_fn(lambda c, p, h, d, n: p['no such key'], names)


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
