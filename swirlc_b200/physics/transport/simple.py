"""Constant-viscosity transport (reference: physics/transport/simple.py:30-107).

kinematic viscosity nu and Prandtl number pr; mu = nu*rho and
kappa = cp*mu/pr are formed inside the viscous-flux kernel.
"""


class TransportSimple:

  def __init__(self, cfg):
    self._nu = cfg.transport_parameters['nu']
    self._pr = cfg.transport_parameters['pr']

  @property
  def nu(self) -> float:
    return float(self._nu)

  @property
  def pr(self) -> float:
    return float(self._pr)
