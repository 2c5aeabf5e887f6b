"""CPU: the z-slab oracle (tests/slab_oracle.py) equals the whole-grid
oracle bit for bit on the slabs' interiors, for a periodic grid, a grid
with z walls and gravity, and the same with hydrostatic helper states; so
the full-size GPU parity tests compare against the reference path
restated, not against an approximation of it."""

import numpy as np
import pytest

from oracle import swirlc_oracle as orc
from tests import slab_oracle

KEYS = ('halo_width', 'dx', 'dy', 'dz', 'interpolation_scheme',
        'numeric_flux_scheme', 'include_diffusion', 'transport_parameters',
        'muscl_limiter', 'x', 'y', 'z', 'bc', 'g', 'source_functions',
        'time_integration_scheme')


@pytest.mark.parametrize('case', ['kh', 'bubble', 'bubble_helper'])
def test_slabs_equal_whole_grid(case):
  from swirlc_b200 import configs
  if case == 'kh':
    uc, st = configs.kelvin_helmholtz(n=24, nu=1e-3)
    helper, slabs, dt = None, [(0, 8), (8, 16), (16, 24)], 1e-3
  else:
    uc, st = configs.buoyant_bubble(nx=12, ny=10, nz=32, lz=100.0)
    helper = (configs.buoyant_bubble_reference_states(12, 10, 32, lz=100.0)
              if case == 'bubble_helper' else None)
    slabs, dt = [(0, 6), (10, 20), (26, 32)], 0.05
  ocfg = orc.make_cfg(**{k: uc[k] for k in KEYS if k in uc})
  s = {k: v.astype(np.float32) for k, v in st.items()}
  hp = ({k: v.astype(np.float32) for k, v in helper.items()}
        if helper else None)
  full = orc.rk3(s, np.float32(dt), lambda u: orc.rhs(u, ocfg, hp))
  res = slab_oracle.one_step(ocfg, st, dt, slabs, helper=helper, procs=2)
  hw = 3
  for (z0, z1), r in zip(slabs, res):
    for k in full:
      np.testing.assert_array_equal(r[k], full[k][z0 + hw:z1 + hw, hw:-hw,
                                                   hw:-hw], err_msg=(z0, k))
