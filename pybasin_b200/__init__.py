"""B200-native fused Dopri5 + steady-state-feature integrator for basin stability.

Drop-in pieces for the reference's pipeline:

* :class:`B200Dopri5Solver` — a ``SolverProtocol`` solver (replaces ``TorchDiffEqSolver``),
* :class:`FusedFeatureExtractor` — the ``TorchFeatureExtractor`` API over in-kernel statistics,
* :func:`register_system` — map an ODE class to a built-in device right-hand side,
* :class:`pybasin_b200.rhs.ExpressionODE` — a user ODE compiled at run time.
"""

from pybasin_b200.features import FrictionFeatureExtractor, FusedFeatureExtractor, impute_extreme
from pybasin_b200.odes import (
    DuffingODE,
    FrictionODE,
    LinearODE,
    LorenzODE,
    PendulumODE,
    register_system,
    resolve_system,
)
from pybasin_b200.solver import B200Dopri5Solver, IntegrationResult

__all__ = [
    "B200Dopri5Solver",
    "IntegrationResult",
    "FusedFeatureExtractor",
    "impute_extreme",
    "register_system",
    "resolve_system",
    "PendulumODE",
    "DuffingODE",
    "LorenzODE",
    "LinearODE",
    "FrictionODE",
    "FrictionFeatureExtractor",
]
