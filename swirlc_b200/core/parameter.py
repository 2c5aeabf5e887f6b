"""Simulation configuration (reference: core/parameter.py:28-255).

`SwirlCParameters(user_cfg)` deep-copies the same default dictionary as the
reference and sets every key as an attribute, so a user cfg dict written for
the reference builds the same object. Keys this implementation adds are
optional and default to the reference's behaviour:

  muscl_limiter  'van_leer' | 'mc' | 'minmod' | 'minmod3' (limiter of the
                 MUSCL scheme; 'minmod3' is the reference prototype's slope)
  cfl            > 0 turns on the device CFL time step (else cfg.dt is used)
  t_end          > 0 clamps the last CFL step to end at t_end
"""

import copy
import os
from typing import Any, Dict, Optional

import numpy as np
import yaml

from swirlc_b200.boundary import bc_types
from swirlc_b200.common import types
from swirlc_b200.numerics import kernel_op_types


def _get_cell_center_coordinates(start: float, stop: float,
                                 n_cells: int) -> np.ndarray:
  xx = np.linspace(start, stop, n_cells + 1, dtype=types.NP_DTYPE)
  xx = xx[:-1] + 0.5 * np.diff(xx)[0]
  return xx


_XX = _get_cell_center_coordinates(0.0, 1.0, 10)
_DX = np.diff(_XX)[0]

_DEFAULT_OPTIONS = {
    'apply_preprocess': False,
    'apply_postprocess': False,
    'states_to_file': None,
    'states_from_file': None,
    'cx': 1,
    'cy': 1,
    'cz': 1,
    'use_3d_tf_tensor': False,
    'halo_width': 3,
    'nx': 10,
    'ny': 10,
    'nz': 10,
    'core_nx': 10,
    'core_ny': 10,
    'core_nz': 10,
    'lx': 1.0,
    'ly': 1.0,
    'lz': 1.0,
    'x': _XX,
    'dx': _DX,
    'y': _XX,
    'dy': _DX,
    'z': _XX,
    'dz': _DX,
    'g': {'x': 0.0, 'y': 0.0, 'z': 0.0},
    'start_step': 0,
    'num_steps': 50,
    'num_cycles': 5,
    'dt': 1.0e-3,
    'solver': 'compressible_navier_stokes',
    'interpolation_scheme': 'WENO_5',
    'numeric_flux_scheme': 'HLL',
    'include_diffusion': False,
    'time_integration_scheme': 'rk3',
    'source_functions': None,
    'kernel_op_type': kernel_op_types.KernelOpType.KERNEL_OP_SLICE.value,
    'kernel_size': 8,
    'thermodynamics_model': 'generic',
    'p_0': 101325.0,
    'transport_model': 'simple',
    'transport_parameters': {'nu': 1.0e-4, 'pr': 0.7},
    'nu': 1e-1,
    'nu_t': None,
    'conservative_variable_names': list(types.BASE_CONSERVATIVE),
    'primitive_variable_names': list(types.BASE_PRIMITIVES),
    'additional_state_names': [],
    'helper_variable_names': [],
    'debug_variables': [],
    'bc': {
        'cell_averages': {
            var_name: {
                dim: {
                    0: (bc_types.BoundaryCondition.PERIODIC,),
                    1: (bc_types.BoundaryCondition.PERIODIC,),
                } for dim in types.DIMS
            } for var_name in types.BASE_CONSERVATIVE
        }
    },
    # Keys added by this implementation (see module docstring).
    'muscl_limiter': 'mc',
    'cfl': 0.0,
    't_end': 0.0,
}


class _KernelOpStub:
  """Stands in for swirl_lm's ApplyKernelOp: stencils run as CUDA kernels."""

  def __init__(self, kind: str):
    self.kind = kind

  def __repr__(self):
    return f'KernelOp({self.kind})'


class SwirlCParameters:
  """The simulation context object (parameter.py:134-248)."""

  def __init__(self, user_cfg: Optional[Dict[str, Any]] = None):
    self._simulation_cfg = copy.deepcopy(_DEFAULT_OPTIONS)
    if user_cfg:
      for key, val in user_cfg.items():
        self._simulation_cfg[key] = val
    for key, val in self._simulation_cfg.items():
      setattr(self, key, val)
    valid = {t.value for t in kernel_op_types.KernelOpType}
    if self.kernel_op_type not in valid:
      raise ValueError('Unknown kernel operator {}'.format(self.kernel_op_type))
    self.kernel_op = _KernelOpStub(self.kernel_op_type)

  def save_to_file(self, prefix: str) -> None:
    """Saves the configuration dictionary as YAML (parameter.py:250-255)."""
    output_dir, _ = os.path.split(prefix)
    if output_dir:
      os.makedirs(output_dir, exist_ok=True)
    with open(f'{prefix}_swirl_c_cfg.yml', 'w') as f:
      yaml.dump(self._simulation_cfg, f, default_flow_style=False)

  @classmethod
  def load_from_file(cls, path: str) -> 'SwirlCParameters':
    """Rebuilds the parameters from a file written by `save_to_file` (the
    file name, or the prefix given to `save_to_file`)."""
    if not path.endswith('.yml'):
      path = f'{path}_swirl_c_cfg.yml'
    with open(path) as f:
      user_cfg = yaml.load(f, Loader=_CfgLoader)
    if not isinstance(user_cfg, dict):
      raise ValueError(f'{path} does not hold a configuration dictionary.')
    return cls(user_cfg)


class _CfgLoader(yaml.SafeLoader):
  """Safe YAML plus the Python tags that `yaml.dump` writes for a
  configuration: tuples, NumPy arrays, scalars and dtypes (in their pickle
  form) and the BoundaryCondition enum (of either package). Any other Python
  tag is an error: no other object is ever constructed."""


_NP_RECONSTRUCT = ('numpy._core.multiarray._reconstruct',
                   'numpy.core.multiarray._reconstruct')
_NP_SCALAR = ('numpy._core.multiarray.scalar', 'numpy.core.multiarray.scalar')


def _yaml_tuple(loader, node):
  return tuple(loader.construct_sequence(node, deep=True))


def _yaml_name(loader, suffix, node):
  del loader, node
  if suffix != 'numpy.ndarray':
    raise yaml.constructor.ConstructorError(
        None, None, f'python/name:{suffix} is not allowed in a configuration')
  return np.ndarray


def _np_dtype(args, state):
  dt = np.dtype(args[0])
  if state is not None and len(state) > 1 and state[1] in ('<', '>'):
    dt = dt.newbyteorder(state[1])
  return dt


def _yaml_apply(loader, suffix, node):
  if isinstance(node, yaml.SequenceNode):
    args, state = loader.construct_sequence(node, deep=True), None
  else:
    m = loader.construct_mapping(node, deep=True)
    args, state = m.get('args', []), m.get('state')
  module, _, name = suffix.rpartition('.')
  if name == 'BoundaryCondition' and module.endswith('bc_types'):
    return bc_types.BoundaryCondition(args[0])
  if suffix == 'numpy.dtype':
    return _np_dtype(args, state)
  if suffix in _NP_RECONSTRUCT and state is not None:
    _, shape, dtype, fortran, raw = state
    arr = np.frombuffer(raw, dtype=dtype)
    return arr.reshape(shape, order='F' if fortran else 'C').copy()
  if suffix in _NP_SCALAR:
    return np.frombuffer(args[1], dtype=args[0])[0]
  raise yaml.constructor.ConstructorError(
      None, None, f'python/object/apply:{suffix} is not allowed in a '
      'configuration', node.start_mark)


_CfgLoader.add_constructor('tag:yaml.org,2002:python/tuple', _yaml_tuple)
_CfgLoader.add_multi_constructor('tag:yaml.org,2002:python/name:', _yaml_name)
_CfgLoader.add_multi_constructor('tag:yaml.org,2002:python/object/apply:',
                                 _yaml_apply)
