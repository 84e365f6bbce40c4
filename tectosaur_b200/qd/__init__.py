"""Quasidynamic rate-and-state fault models on the device (reference:
tectosaur/qd: FullspaceModel, Integrator, the rate-state Newton solve and
the aging law)."""
siay = 60 * 60 * 24 * 365.25

from .model import FullspaceModel, aging_law, build_elastic_op, calc_derived_constants  # noqa: E402
from .integrator import Integrator  # noqa: E402
from .rk23 import RK23  # noqa: E402
