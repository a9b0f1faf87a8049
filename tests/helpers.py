"""Shared case definitions for the tests (the reference's case-study setups).

Pendulum: case_studies/pendulum/setup_pendulum_system.py:18-75.
Duffing:  case_studies/duffing_oscillator/setup_duffing_oscillator_system.py:11-70.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from oracle import oracle as O


@dataclass(frozen=True)
class Case:
    name: str
    oracle_sys: int
    params: tuple[float, ...]
    lo: tuple[float, ...]
    hi: tuple[float, ...]
    t_span: tuple[float, float]
    t_eval: tuple[float, float]
    t_steps: int
    time_steady: float
    # (state, oracle feature kind, param, reference feature name)
    features: tuple[tuple[int, int, float, str], ...]
    templates: tuple[tuple[float, ...], ...]
    classes: tuple[str, ...]
    rtol: float = 1e-8
    atol: float = 1e-6
    extra: dict = field(default_factory=dict)

    def save_ts(self) -> torch.Tensor:
        return torch.linspace(self.t_eval[0], self.t_eval[1], self.t_steps, dtype=torch.float32).double()

    def win_begin(self) -> int:
        s = self.save_ts().numpy()
        return int(np.nonzero(s >= self.time_steady)[0][0])


PENDULUM = Case(
    name="pendulum",
    oracle_sys=O.SYS_PENDULUM,
    params=(0.1, 0.5, 1.0),
    lo=(-np.pi + np.arcsin(0.5), -10.0),
    hi=(np.pi + np.arcsin(0.5), 10.0),
    t_span=(0.0, 1000.0),
    t_eval=(0.0, 1000.0),
    t_steps=1000,
    time_steady=950.0,
    features=((1, 9, 0.0, "log_delta"),),
    templates=((0.4, 0.0), (2.7, 0.0)),
    classes=("FP", "LC"),
)

DUFFING = Case(
    name="duffing",
    oracle_sys=O.SYS_DUFFING,
    params=(0.08, 1.0, 0.2),
    lo=(-1.0, -0.5),
    hi=(1.0, 1.0),
    t_span=(0.0, 1000.0),
    t_eval=(900.0, 1000.0),
    t_steps=5000,
    time_steady=900.0,
    features=((0, 5, 0.0, "maximum"), (0, 2, 0.0, "standard_deviation")),
    templates=((-0.21, 0.02), (1.05, 0.77), (-0.67, 0.02), (-0.46, 0.30), (-0.43, 0.12)),
    classes=tuple(f"$\\bar{{y}}_{i}$" for i in range(1, 6)),
)


def seeded_ics(case: Case, n: int, seed: int = 42) -> torch.Tensor:
    """UniformRandomSampler.sample after torch.manual_seed (src/pybasin/sampler.py:56-65)."""
    torch.manual_seed(seed)
    lo = torch.tensor(case.lo, dtype=torch.float32)
    hi = torch.tensor(case.hi, dtype=torch.float32)
    return torch.rand(n, len(case.lo)) * (hi - lo) + lo


def oracle_case_features(case: Case, y0: np.ndarray, rtol: float | None = None, atol: float | None = None):
    """FP64 oracle features of ``y0`` and of the case templates."""
    save = case.save_ts().numpy()
    feats = [(f[0], f[1], f[2]) for f in case.features]
    kw = dict(win_begin=case.win_begin(), features=feats)
    r = O.solve_batch(case.oracle_sys, y0, np.array([case.params]), save, (case.t_span[0], float(save[-1])),
                      rtol or case.rtol, atol or case.atol, **kw)
    rt = O.solve_batch(case.oracle_sys, np.array(case.templates), np.array([case.params]), save,
                       (case.t_span[0], float(save[-1])), rtol or case.rtol, atol or case.atol, **kw)
    return r["features"], rt["features"], r


def impute(f: np.ndarray) -> np.ndarray:
    return np.nan_to_num(f, nan=1e10, posinf=1e10, neginf=-1e10)


def knn_labels(template_features: np.ndarray, features: np.ndarray) -> np.ndarray:
    """The reference's KNeighborsClassifier(n_neighbors=1) on FP32 features."""
    from sklearn.neighbors import KNeighborsClassifier

    knn = KNeighborsClassifier(n_neighbors=1)
    knn.fit(impute(template_features).astype(np.float32), np.arange(len(template_features)))
    return knn.predict(impute(features).astype(np.float32))
