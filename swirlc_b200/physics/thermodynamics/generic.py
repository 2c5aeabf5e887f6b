"""Ideal-gas thermodynamics (reference: physics/thermodynamics/generic.py).

The pressure, enthalpy, sound-speed and potential-energy formulas of
generic.py:27-439 are evaluated inside the CUDA kernels
(swirlc_b200/csrc/swc_physics.cuh). This class keeps the reference's option
validation for callers that select options by name.
"""

from swirlc_b200.common import types


class ThermodynamicsGeneric:
  """generic.py:24-440 (configuration side)."""

  SOUND_SPEED_OPTIONS = (types.E, types.H, 'p_rho')

  def check_sound_speed_option(self, opt: str) -> None:
    if opt not in self.SOUND_SPEED_OPTIONS:
      raise ValueError(
          f'"{opt}" is not a valid option for sound speed. Available options'
          f' are "{types.E}", "{types.H}", "p_rho".')
