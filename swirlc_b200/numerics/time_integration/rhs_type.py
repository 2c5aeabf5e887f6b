"""RHS callable type (reference: numerics/time_integration/rhs_type.py:22-29)."""

from typing import Callable

from swirlc_b200.common import types

RHS = Callable[[object, types.FlowFieldMap, types.FlowFieldMap],
               types.FlowFieldMap]
