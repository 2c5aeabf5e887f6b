"""Face interpolation (reference: numerics/interpolation.py and the
swirl_lm interpolation functions it calls,
compressible_navier_stokes.py:581-589).

weno(v, dim, k) and flux_limiter(v, dim, limiter_type) return (neg, pos) at
face i-1/2: neg reconstructed from the left cell i-1, pos from cell i. WENO
uses the Jiang-Shu weights alpha_r = d_r / (1e-6 + beta_r)^2 (k = 3: WENO5,
k = 2: WENO3); the flux limiter is a slope-limited MUSCL reconstruction.
Points whose stencil leaves the array are set to 0.
"""

import enum

from swirlc_b200 import _native as nat
from swirlc_b200.numerics import _pointwise


class FluxLimiterType(enum.Enum):
  """MUSCL is the monotonized-central limiter of van Leer's MUSCL scheme."""
  MUSCL = 'mc'
  VAN_LEER = 'van_leer'
  MINMOD = 'minmod'
  # The reference prototype's slope (demo/swirl_c_prototype.ipynb `muscl`):
  # minmod of the central, forward and backward differences.
  MINMOD3 = 'minmod3'


_LIM = {'van_leer': nat.SWC_LIM_VAN_LEER, 'mc': nat.SWC_LIM_MC,
        'minmod': nat.SWC_LIM_MINMOD, 'minmod3': nat.SWC_LIM_MINMOD3}


def weno(v, dim: str, k: int = 3):
  if k == 3:
    return _pointwise.reconstruct(v, dim, nat.SWC_WENO5)
  if k == 2:
    return _pointwise.reconstruct(v, dim, nat.SWC_WENO3)
  raise NotImplementedError(f'WENO with k = {k} is not implemented.')


def flux_limiter(v, dim: str, limiter_type=FluxLimiterType.VAN_LEER):
  key = getattr(limiter_type, 'value', limiter_type)
  if key not in _LIM:
    raise NotImplementedError(f'Flux limiter "{limiter_type}" is not '
                              'implemented.')
  return _pointwise.reconstruct(v, dim, nat.SWC_MUSCL, _LIM[key])


def linear_interpolation(f, dim: str, kernel_op=None):
  """interpolation.py:21-53: 0.5 * (f[i-1] + f[i]) on face i-1/2."""
  del kernel_op
  return _pointwise.stencil(f, 3, dim, 1.0)
