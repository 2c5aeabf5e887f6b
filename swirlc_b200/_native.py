"""ctypes binding of the C-ABI library libswirlc_b200.so (include/swirlc_b200.h).

The library is built in-tree (swirlc_b200/lib) by `python -m swirlc_b200.build`.
There is no fallback: if the library or a CUDA device is missing, every
compute entry point raises.
"""

from __future__ import annotations

import ctypes
import os
import threading
from typing import Optional, Sequence

import torch

# SWIRLC_B200_LIB overrides the in-tree library path (e.g. an alternative
# build of the same sources).
_LIB_PATH = os.environ.get('SWIRLC_B200_LIB') or os.path.join(
    os.path.dirname(os.path.abspath(__file__)), 'lib', 'libswirlc_b200.so')

SWC_OK = 0
SWC_ERR_ARG = -1
SWC_ERR_UNSUPPORTED = -2
SWC_ERR_LAUNCH = -3
SWC_ERR_TIMEOUT = -4
SWC_ERR_NONFINITE = -5

SWC_F32, SWC_F64 = 0, 1
SWC_WENO5, SWC_WENO3, SWC_MUSCL, SWC_NODE = 0, 1, 2, 3
SWC_LIM_VAN_LEER, SWC_LIM_MC, SWC_LIM_MINMOD, SWC_LIM_MINMOD3 = 0, 1, 2, 3
SWC_HLL, SWC_HLLC = 0, 1
SWC_BC_PERIODIC, SWC_BC_DIRICHLET, SWC_BC_NEUMANN, SWC_BC_NONE = 0, 1, 2, 4
SWC_OUT_RHS, SWC_OUT_EULER, SWC_OUT_CONVEX, SWC_OUT_AVERAGE = 0, 1, 2, 3
SWC_MAX_FIELDS = 8
SWC_VISC_FLUX, SWC_VISC_STRAIN, SWC_VISC_STRESS, SWC_VISC_HEAT = 0, 1, 2, 3

# Every symbol include/swirlc_b200.h declares.
EXPORTED = (
    'swc_abi_version', 'swc_last_error', 'swc_launch_count', 'swc_halo_fill',
    'swc_rk_stage', 'swc_cfl_reduce', 'swc_clock_begin_step',
    'swc_clock_end_step', 'swc_clock_status', 'swc_reconstruct', 'swc_riemann_flux',
    'swc_wave_speeds', 'swc_stencil', 'swc_viscous_terms', 'swc_rk_combine',
    'swc_rk_step',
    'swc_rk_step_noalloc', 'swc_batch_step', 'swc_rk_stage_ext',
    'swc_rk_stage_vjp',
    'swc_rk_step_vjp',
)

# Built-in work space of swc_rk_step_noalloc (SWC_NOALLOC_MAX_BYTES).
SWC_NOALLOC_MAX_BYTES = 64 << 20


class SwcGrid(ctypes.Structure):
  _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32),
              ('nz', ctypes.c_int32), ('halo', ctypes.c_int32),
              ('sx', ctypes.c_int64), ('sz', ctypes.c_int64),
              ('dx', ctypes.c_double), ('dy', ctypes.c_double),
              ('dz', ctypes.c_double)]


class SwcScheme(ctypes.Structure):
  _fields_ = [('dtype', ctypes.c_int32), ('interp', ctypes.c_int32),
              ('limiter', ctypes.c_int32), ('riemann', ctypes.c_int32),
              ('diffusion', ctypes.c_int32), ('nscalars', ctypes.c_int32),
              ('gravity_mask', ctypes.c_int32), ('zseg', ctypes.c_int32),
              ('tile', ctypes.c_int32), ('reserved', ctypes.c_int32),
              ('nu', ctypes.c_double), ('pr', ctypes.c_double),
              ('g', ctypes.c_double * 3), ('pe_axis', ctypes.c_void_p * 3)]


class SwcBC(ctypes.Structure):
  _fields_ = [('kind', ctypes.c_int32), ('per_layer', ctypes.c_int32),
              ('value', ctypes.c_double), ('planes', ctypes.c_void_p)]


class SwcFieldBC(ctypes.Structure):
  _fields_ = [('via_primitive', ctypes.c_int32), ('reserved', ctypes.c_int32),
              ('side', (SwcBC * 2) * 3)]


class SwcClock(ctypes.Structure):
  _fields_ = [('t', ctypes.c_double), ('dt', ctypes.c_double),
              ('dtmin', ctypes.c_double), ('cfl', ctypes.c_double),
              ('t_end', ctypes.c_double), ('step', ctypes.c_int64)]


SWC_MAX_OVERRIDES = 8
# Scratch buffers of swc_rk_stage_vjp (SWC_VJP_SCRATCH).
SWC_VJP_SCRATCH = 79
SWC_FACE_PRIMITIVE, SWC_FACE_CONSERVATIVE = 0, 1
SWC_FLUX_CONVECTIVE, SWC_FLUX_DIFFUSIVE, SWC_FLUX_TOTAL = 0, 1, 2


class SwcOverride(ctypes.Structure):
  _fields_ = [('var', ctypes.c_int32), ('mode', ctypes.c_int32),
              ('value', ctypes.c_double), ('plane', ctypes.c_void_p)]


class SwcStageExt(ctypes.Structure):
  _fields_ = [('p_ref', ctypes.c_void_p), ('rho_ref', ctypes.c_void_p),
              ('boundary', (ctypes.c_int32 * 2) * 3),
              ('nface', (ctypes.c_int32 * 2) * 3),
              ('nflux', (ctypes.c_int32 * 2) * 3),
              ('reserved', ctypes.c_int32),
              ('face', ((SwcOverride * SWC_MAX_OVERRIDES) * 2) * 3),
              ('flux', ((SwcOverride * SWC_MAX_OVERRIDES) * 2) * 3)]


class SwcBatchMember(ctypes.Structure):
  _fields_ = [('grid', SwcGrid), ('u', ctypes.c_void_p * 5),
              ('work', ctypes.c_void_p * 10), ('pe_axis', ctypes.c_void_p * 3),
              ('bcs', SwcFieldBC * 5), ('clock', ctypes.c_void_p),
              ('tile', ctypes.c_int32), ('zseg', ctypes.c_int32)]


_lib: Optional[ctypes.CDLL] = None
_lock = threading.Lock()


def lib_path() -> str:
  return _LIB_PATH


def load(require_cuda: bool = True) -> ctypes.CDLL:
  """Loads the library; raises if it is missing (no fallback path exists)."""
  global _lib
  if require_cuda and not torch.cuda.is_available():
    raise RuntimeError('swirlc_b200 needs a CUDA device; none is visible.')
  with _lock:
    if _lib is None:
      if not os.path.exists(_LIB_PATH):
        raise RuntimeError(
            f'swirlc_b200 native library not found at {_LIB_PATH}; build it '
            'with `python -m swirlc_b200.build`.')
      lib = ctypes.CDLL(_LIB_PATH)
      vp = ctypes.c_void_p
      i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
      pp = ctypes.POINTER(ctypes.c_void_p)
      lib.swc_abi_version.restype = ctypes.c_int
      lib.swc_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
      lib.swc_launch_count.restype = ctypes.c_int64
      lib.swc_halo_fill.argtypes = [ctypes.POINTER(SwcGrid), i32, i32, pp,
                                    ctypes.POINTER(SwcFieldBC), i32, vp]
      lib.swc_rk_stage.argtypes = [ctypes.POINTER(SwcGrid),
                                   ctypes.POINTER(SwcScheme), pp, pp, pp, i32,
                                   dbl, dbl, vp, vp, vp]
      lib.swc_cfl_reduce.argtypes = [ctypes.POINTER(SwcGrid),
                                     ctypes.POINTER(SwcScheme), pp, vp, vp]
      lib.swc_clock_begin_step.argtypes = [vp, vp]
      lib.swc_clock_end_step.argtypes = [vp, vp]
      lib.swc_clock_status.argtypes = [vp, vp]
      lib.swc_reconstruct.argtypes = [ctypes.POINTER(SwcGrid), i32, i32, i32,
                                      i32, vp, vp, vp, vp]
      lib.swc_riemann_flux.argtypes = [i64, i32, i32, i32, i32, pp, pp, vp, vp,
                                       vp, pp, vp]
      lib.swc_wave_speeds.argtypes = [i64, i32, i32, pp, pp, vp, vp, vp, vp,
                                      vp]
      lib.swc_stencil.argtypes = [ctypes.POINTER(SwcGrid), i32, i32, i32, dbl,
                                  vp, vp, vp]
      lib.swc_viscous_terms.argtypes = [ctypes.POINTER(SwcGrid), i32, i32, pp,
                                        pp, dbl, dbl, pp, vp]
      lib.swc_rk_combine.argtypes = [i64, i32, i32, dbl, dbl, vp, vp, vp, vp,
                                     vp, vp]
      lib.swc_rk_step.argtypes = [ctypes.POINTER(SwcGrid),
                                  ctypes.POINTER(SwcScheme),
                                  ctypes.POINTER(SwcFieldBC), i32, pp, pp, vp,
                                  vp]
      lib.swc_rk_stage_ext.argtypes = [ctypes.POINTER(SwcGrid),
                                       ctypes.POINTER(SwcScheme),
                                       ctypes.POINTER(SwcStageExt), pp, pp, pp,
                                       i32, dbl, dbl, vp, vp, vp]
      lib.swc_rk_stage_vjp.argtypes = [ctypes.POINTER(SwcGrid),
                                       ctypes.POINTER(SwcScheme),
                                       ctypes.POINTER(SwcFieldBC), pp, pp, dbl,
                                       dbl, pp, dbl, pp, dbl, pp, vp, pp, vp]
      lib.swc_rk_step_vjp.argtypes = [ctypes.POINTER(SwcGrid),
                                      ctypes.POINTER(SwcScheme),
                                      ctypes.POINTER(SwcFieldBC), i32, pp, dbl,
                                      pp, pp, pp, vp, pp, vp]
      lib.swc_batch_step.argtypes = [ctypes.POINTER(SwcScheme), i32, i32,
                                     ctypes.POINTER(SwcBatchMember), vp]
      lib.swc_rk_step_noalloc.argtypes = [ctypes.POINTER(SwcGrid),
                                          ctypes.POINTER(SwcScheme),
                                          ctypes.POINTER(SwcFieldBC), i32, pp,
                                          vp, vp]
      for name in EXPORTED:
        fn = getattr(lib, name)
        if fn.restype is ctypes.c_int and name not in ('swc_abi_version',):
          fn.restype = ctypes.c_int
      _lib = lib
  return _lib


def last_error() -> str:
  lib = load(require_cuda=False)
  buf = ctypes.create_string_buffer(1024)
  lib.swc_last_error(buf, len(buf))
  return buf.value.decode()


def check(rc: int, what: str = '') -> None:
  """Maps a C status to the exception types the reference raises."""
  if rc == SWC_OK:
    return
  msg = last_error()
  if what:
    msg = f'{what}: {msg}'
  if rc == SWC_ERR_ARG:
    raise ValueError(msg)
  if rc == SWC_ERR_UNSUPPORTED:
    raise NotImplementedError(msg)
  if rc == SWC_ERR_NONFINITE:
    raise FloatingPointError(msg)
  raise RuntimeError(msg)


def launch_count() -> int:
  return int(load(require_cuda=False).swc_launch_count())


def stream_ptr(stream: Optional[torch.cuda.Stream] = None) -> int:
  s = stream if stream is not None else torch.cuda.current_stream()
  return int(s.cuda_stream)


def ptr_array(tensors: Sequence[Optional[torch.Tensor]]):
  arr = (ctypes.c_void_p * max(1, len(tensors)))()
  for i, t in enumerate(tensors):
    arr[i] = None if t is None else t.data_ptr()
  return arr


def addr_array(addrs: Sequence[Optional[int]]):
  """A void* array from raw device addresses (None for NULL)."""
  arr = (ctypes.c_void_p * max(1, len(addrs)))()
  for i, a in enumerate(addrs):
    arr[i] = a
  return arr


def dtype_code(dtype: torch.dtype) -> int:
  if dtype == torch.float32:
    return SWC_F32
  if dtype == torch.float64:
    return SWC_F64
  raise ValueError(f'Unsupported dtype {dtype}; use float32 or float64.')
