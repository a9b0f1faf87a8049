"""ODE systems the B200 solver integrates, and how reference ODE objects map to them.

The solver accepts any object with the reference's ``ODESystemProtocol``
(src/pybasin/protocols.py:70-113): a ``params`` mapping whose value order is the
column order of the parameter array (``params_to_array``,
src/pybasin/solvers/torch_ode_system.py:57-66).  The right-hand side runs as a
templated device functor; which one is chosen by (in order):

1. an attribute ``b200_system`` on the object or its class (a name or id),
2. the class name, for the reference's case-study systems
   (``PendulumODE``/``PendulumJaxODE``/``PendulumNumpyODE``, ``DuffingODE``...),
3. names registered with :func:`register_system`.

An object with ``b200_system = "user"`` (``pybasin_b200.rhs.ExpressionODE``)
carries its own right-hand side as C expressions, compiled at run time.

The classes defined here are minimal ODE systems with the reference's
interface for users who do not have pybasin installed.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np
import torch

from pybasin_b200 import _lib as L

SYSTEM_IDS: dict[str, int] = {
    "linear": L.SYS_LINEAR,
    "pendulum": L.SYS_PENDULUM,
    "duffing": L.SYS_DUFFING,
    "lorenz": L.SYS_LORENZ,
    "lorenz_masked": L.SYS_LORENZ_MASKED,
    "rossler_network": L.SYS_ROSSLER_NET,
    "friction": L.SYS_FRICTION,
    "user": L.SYS_USER,  # expressions compiled at run time (pybasin_b200.rhs.ExpressionODE)
}

# reference class name -> system (case_studies/*/*_ode.py, tests/unit/solvers/test_solver.py)
_CLASS_MAP: dict[str, str] = {
    "PendulumODE": "pendulum",
    "PendulumJaxODE": "pendulum",
    "PendulumNumpyODE": "pendulum",
    "DuffingODE": "duffing",
    "DuffingJaxODE": "duffing",
    "DuffingNumpyODE": "duffing",
    "LorenzODE": "lorenz_masked",  # torch variant freezes at |y|>=200 (lorenz_ode.py:52-64)
    "LorenzJaxODE": "lorenz",
    "LorenzNumpyODE": "lorenz",
    "ExponentialDecayODE": "linear",
    "ExponentialDecayNumpyODE": "linear",
    "LinearODE": "linear",
    "RosslerNetworkJaxODE": "rossler_network",
    "RosslerNetworkODE": "rossler_network",
    "FrictionODE": "friction",
    "FrictionJaxODE": "friction",
}

_DIMS: dict[int, tuple[int, ...]] = {
    L.SYS_LINEAR: (1, 2, 3, 4),
    L.SYS_PENDULUM: (2,),
    L.SYS_DUFFING: (2,),
    L.SYS_LORENZ: (3,),
    L.SYS_LORENZ_MASKED: (3,),
    L.SYS_ROSSLER_NET: tuple(3 * n for n in range(1, 129)),
    L.SYS_FRICTION: (2,),
    L.SYS_USER: tuple(range(1, L.MAX_USER_DIM + 1)),
}


def register_system(name_or_cls: str | type, system: str | int) -> None:
    """Map an ODE class (or class name) to a built-in device right-hand side."""
    key = name_or_cls if isinstance(name_or_cls, str) else name_or_cls.__name__
    _CLASS_MAP[key] = system if isinstance(system, str) else _name_of(system)


def _name_of(system_id: int) -> str:
    for k, v in SYSTEM_IDS.items():
        if v == system_id:
            return k
    raise ValueError(f"unknown system id {system_id}")


@dataclass(frozen=True)
class SystemSpec:
    system: int
    dim: int
    params: np.ndarray  # (n_params,) float64 default parameters


def params_array(ode_system: Any) -> np.ndarray:
    """Default parameter row of ``ode_system`` in TypedDict order."""
    p = getattr(ode_system, "params", None)
    if isinstance(p, dict) and p:
        return np.asarray([float(v) for v in p.values()], dtype=np.float64)
    to_arr = getattr(ode_system, "params_to_array", None)
    if callable(to_arr):
        return np.asarray(np.asarray(to_arr()), dtype=np.float64).reshape(-1)
    raise ValueError(f"{type(ode_system).__name__} has no params mapping")


def resolve_system(ode_system: Any, dim: int) -> SystemSpec:
    """Identify the device right-hand side for ``ode_system`` at state dimension ``dim``."""
    tag = getattr(ode_system, "b200_system", None)
    if tag is None:
        tag = _CLASS_MAP.get(type(ode_system).__name__)
    if tag is None:
        raise ValueError(
            f"no B200 right-hand side for {type(ode_system).__name__}; set `b200_system` on the class "
            f"or call pybasin_b200.register_system (built-ins: {sorted(SYSTEM_IDS)})"
        )
    sid = tag if isinstance(tag, int) else SYSTEM_IDS[str(tag)]
    if sid == L.SYS_USER and len(getattr(ode_system, "b200_rhs", ())) != dim:
        raise ValueError(f"{type(ode_system).__name__} defines no right-hand side for state dimension {dim}")
    if dim not in _DIMS.get(sid, ()):
        raise ValueError(f"system '{_name_of(sid)}' does not support state dimension {dim}")
    params = params_array(ode_system)
    if params.shape[0] > L.MAX_PARAMS:
        raise ValueError(f"at most {L.MAX_PARAMS} parameters are supported")
    return SystemSpec(sid, dim, params)


# ---------------------------------------------------------------------------
# Minimal ODE systems with the reference interface (torch RHS for host use)
# ---------------------------------------------------------------------------
class ODESystem(torch.nn.Module):
    """Base with the reference's ``ODESystem`` surface (torch_ode_system.py:12-79)."""

    b200_system: str | None = None

    def __init__(self, params: dict[str, float]):
        super().__init__()
        self.params = params

    def ode(self, t: torch.Tensor, y: torch.Tensor, p: torch.Tensor) -> torch.Tensor:  # pragma: no cover
        raise NotImplementedError

    def params_to_array(self) -> torch.Tensor:
        return torch.tensor(list(self.params.values()))

    def forward(self, t: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
        p = getattr(self, "_batched_params", None)
        if p is None:
            p = self.params_to_array()
        return self.ode(t, y, p)

    def get_str(self) -> str:
        return f"{type(self).__name__}({self.params})"


class LinearODE(ODESystem):
    """dy/dt = decay * y."""

    b200_system = "linear"

    def ode(self, t, y, p):
        return p[..., 0:1] * y


class PendulumODE(ODESystem):
    """Damped driven pendulum, params {alpha, T, K} (case_studies/pendulum/pendulum_ode.py)."""

    b200_system = "pendulum"

    def ode(self, t, y, p):
        a, T, K = p[..., 0], p[..., 1], p[..., 2]
        return torch.stack([y[..., 1], -a * y[..., 1] + T - K * torch.sin(y[..., 0])], dim=-1)


class DuffingODE(ODESystem):
    """Forced Duffing, params {delta, k3, A} (case_studies/duffing_oscillator/duffing_ode.py)."""

    b200_system = "duffing"

    def ode(self, t, y, p):
        d, k3, A = p[..., 0], p[..., 1], p[..., 2]
        x = y[..., 0]
        return torch.stack([y[..., 1], -d * y[..., 1] - k3 * x**3 + A * torch.cos(t)], dim=-1)


class LorenzODE(ODESystem):
    """Lorenz, params {sigma, r, b}; stop with ``unbounded_threshold`` on the solver."""

    b200_system = "lorenz"

    def ode(self, t, y, p):
        s, r, b = p[..., 0], p[..., 1], p[..., 2]
        x, yy, z = y[..., 0], y[..., 1], y[..., 2]
        return torch.stack([s * (yy - x), r * x - x * z - yy, x * yy - b * z], dim=-1)


class FrictionODE(ODESystem):
    """Friction oscillator, params {v_d, xi, musd, mud, muv, v0}
    (case_studies/friction/friction_ode.py:32-75)."""

    b200_system = "friction"

    def ode(self, t, y, p):
        vd, xi, musd, mud, muv, v0 = (p[..., i] for i in range(6))
        disp, vel = y[..., 0], y[..., 1]
        vrel = vel - vd
        f_fric = mud + mud * (musd - 1.0) * torch.exp(-torch.abs(vrel) / v0) + muv * torch.abs(vrel) / v0
        slip = torch.abs(vrel) > 1e-4
        trans = torch.abs(disp + 2 * xi * vel) > mud * musd
        slip_vel = -disp - 2 * xi * vel - torch.tanh(50 * vrel) * f_fric
        trans_vel = -disp - 2 * xi * vel + mud * musd * torch.tanh(50 * f_fric)
        stick_vel = -(vel - vd)
        return torch.stack([torch.where(slip | trans, vel, vd),
                            torch.where(slip, slip_vel, torch.where(trans, trans_vel, stick_vel))], dim=-1)
