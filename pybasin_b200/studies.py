"""Parameter studies of the case studies at their full sizes, each one launch.

The reference runs a parameter study as B ICs integrated against every
parameter row (IC-major expansion, src/pybasin/solvers/base.py:155-159,
src/pybasin/basin_stability_study.py:166-178).  Here every IC carries its own
parameter point, so points may have different sample counts, and a whole
study is one integrator launch plus one labelling launch (graph-capturable):

* :func:`pendulum_torque_sweep` — the damped driven pendulum
  (case_studies/pendulum/setup_pendulum_system.py) with the torque T swept over
  ``linspace(0.1, 1.0, 64)``; point p has ``round(exp(U(ln 1e3, ln 5e4)))``
  ICs (``numpy.random.default_rng(42)``), drawn by the reference sampler with
  seed 42 + p over the setup's box; 1-NN on the setup's two templates.
* :func:`lorenz_rho_sweep` — Lorenz sigma = 10, beta = 8/3, rho in {0.5, 15,
  28}, ICs uniform on [-20, 20]^3, trajectories reaching |y| > 1e6 stopped and
  labelled unbounded; classes from the window statistics: the origin, the two
  fixed points C+ / C-, and the butterfly.
* :func:`rossler_coupling_sweep` — the Rössler network (a = b = 0.2, c = 7) on a
  seeded Watts-Strogatz graph (100 nodes, k = 4, p = 0.1) with the coupling K
  over ``linspace(0.05, 0.3, 8)``, ICs uniform on [-15, 15]^2 x [-5, 35] per node,
  labelled synchronised / not / unbounded by the reference classifier's 1.5
  threshold (case_studies/rossler_network/synchronization_classifier.py:36-54,
  setup_rossler_network_system.py:91-105; the reference's rtol 1e-3).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

PENDULUM_BOX = ((-np.pi + np.arcsin(0.5), -10.0), (np.pi + np.arcsin(0.5), 10.0))


def uniform_ics(lo, hi, n: int, seed: int) -> torch.Tensor:
    """UniformRandomSampler.sample after torch.manual_seed(seed) (src/pybasin/sampler.py:56-65)."""
    torch.manual_seed(seed)
    lo_t = torch.tensor(lo, dtype=torch.float32)
    hi_t = torch.tensor(hi, dtype=torch.float32)
    return torch.rand(n, len(lo)) * (hi_t - lo_t) + lo_t


@dataclass
class Study:
    """ICs, the parameter point of each IC, and the parameter rows of a study."""

    y0: torch.Tensor  # (n, S) float32, host
    group: torch.Tensor  # (n,) int32, host
    rows: np.ndarray  # (P, n_params)
    counts: np.ndarray  # (P,) ICs per point


def pendulum_torque_sweep(n_points: int = 64, lo: int = 1_000, hi: int = 50_000, seed: int = 42) -> Study:
    rng = np.random.default_rng(seed)
    T = np.linspace(0.1, 1.0, n_points)
    n_p = np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), n_points))).astype(np.int64)
    y0 = torch.cat([uniform_ics(*PENDULUM_BOX, int(k), seed + p) for p, k in enumerate(n_p)])
    group = torch.cat([torch.full((int(k),), p, dtype=torch.int32) for p, k in enumerate(n_p)])
    rows = np.array([[0.1, t, 1.0] for t in T])
    return Study(y0, group, rows, n_p)


def pendulum_pipeline(precision: str, rows: np.ndarray, device: torch.device):
    """The pendulum case's fused pipeline (log_delta of the velocity on t >= 950,
    1000 saves over [0, 1000], the templates (0.4, 0) FP and (2.7, 0) LC) over the
    study's parameter rows."""
    from pybasin_b200 import B200Dopri5Solver, FusedFeatureExtractor, PendulumODE
    from pybasin_b200.pipeline import BasinStabilityPipeline

    fx = FusedFeatureExtractor(time_steady=950.0, features=None, features_per_state={1: {"log_delta": None}},
                               normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=1000, device=str(device), precision=precision,
                              feature_extractor=fx, schedule="probed" if precision == "mixed" else "plain")
    return BasinStabilityPipeline(PendulumODE({"alpha": 0.1, "T": 0.5, "K": 1.0}), solver, [[0.4, 0.0], [2.7, 0.0]],
                                  ["FP", "LC"], device=device, param_rows=rows)


LORENZ_RHO = (0.5, 15.0, 28.0)
LORENZ_CLASSES = ("origin", "C+", "C-", "butterfly", "unbounded")


def lorenz_rho_sweep(per_point: int = 20_000, seed: int = 42) -> Study:
    y0 = torch.cat([uniform_ics((-20.0,) * 3, (20.0,) * 3, per_point, seed + p) for p in range(len(LORENZ_RHO))])
    group = torch.repeat_interleave(torch.arange(len(LORENZ_RHO), dtype=torch.int32), per_point)
    rows = np.array([[10.0, rho, 8.0 / 3.0] for rho in LORENZ_RHO])
    return Study(y0, group, rows, np.full(len(LORENZ_RHO), per_point))


def lorenz_labels(features: torch.Tensor, status: torch.Tensor) -> torch.Tensor:
    """Classes of LORENZ_CLASSES from (mean x, std x) over the window: a spread
    above 1 is the butterfly, else the sign of the mean picks C+ / C- (|mean x|
    above 1) or the origin; a stopped runaway is unbounded."""
    mean_x, std_x = features[:, 0], features[:, 1]
    lab = torch.where(mean_x > 1.0, 1, torch.where(mean_x < -1.0, 2, 0))
    lab = torch.where(std_x > 1.0, 3, lab)
    from pybasin_b200 import _lib as L

    return torch.where(status == L.TRAJ_UNBOUNDED, 4, lab).to(torch.int32)


def lorenz_solve(study: Study, precision: int, device: torch.device, t1: float = 1000.0):
    """One launch over the whole sweep: window [0.9 t1, t1] with 1000 saves, the
    mean and spread of x, unbounded stop at 1e6."""
    from pybasin_b200 import _lib as L
    from pybasin_b200.engine import FeatureColumn, SolveRequest, solve

    save = torch.linspace(0.9 * t1, t1, 1000, dtype=torch.float32).double()
    req = SolveRequest(system=L.SYS_LORENZ, dim=3, y0=study.y0.to(device), params=torch.tensor(study.rows,
                       device=device), save_ts=save.to(device), t_span=(0.0, t1), rtol=1e-8, atol=1e-6,
                       layout=L.LAYOUT_INDEXED, param_index=study.group.to(device),
                       columns=[FeatureColumn(0, L.FEAT_MEAN), FeatureColumn(0, L.FEAT_STD)], unbounded_thr=1e6,
                       precision=precision, keep_final=False, keep_steps=True,
                       schedule=L.SCHED_PROBED if precision == L.PREC_MIXED else L.SCHED_PLAIN,
                       window_record_cap=4096)  # the butterfly takes ~10^3-10^4 steps in the window
    return solve(req)


ROSSLER_K = tuple(np.linspace(0.05, 0.3, 8).tolist())


def rossler_coupling_sweep(per_point: int = 20_000, seed: int = 42, n_nodes: int = 100) -> tuple[Study, tuple]:
    from pybasin_b200.network import csr_from_edges, watts_strogatz

    lo = (-15.0,) * n_nodes + (-15.0,) * n_nodes + (-5.0,) * n_nodes
    hi = (15.0,) * n_nodes + (15.0,) * n_nodes + (35.0,) * n_nodes
    y0 = torch.cat([uniform_ics(lo, hi, per_point, seed + p) for p in range(len(ROSSLER_K))])
    group = torch.repeat_interleave(torch.arange(len(ROSSLER_K), dtype=torch.int32), per_point)
    rows = np.array([[0.2, 0.2, 7.0, k] for k in ROSSLER_K])
    csr = csr_from_edges(watts_strogatz(n_nodes, 4, 0.1, seed=seed), n_nodes)
    return Study(y0, group, rows, np.full(len(ROSSLER_K), per_point)), csr


def rossler_solve(study: Study, csr: tuple, precision: int, device: torch.device, t1: float = 1000.0):
    """One launch over all couplings: the synchronisation features at t1, unbounded
    stop at 400 (setup_rossler_network_system.py:34-43), the reference's tolerances."""
    from pybasin_b200 import _lib as L
    from pybasin_b200.engine import FeatureColumn, SolveRequest, solve

    dim = study.y0.shape[1]
    req = SolveRequest(system=L.SYS_ROSSLER_NET, dim=dim, y0=study.y0.to(device),
                       params=torch.tensor(study.rows, device=device),
                       save_ts=torch.tensor([t1], dtype=torch.float64, device=device), t_span=(0.0, t1), rtol=1e-3,
                       atol=1e-6, layout=L.LAYOUT_INDEXED, param_index=study.group.to(device),
                       columns=[FeatureColumn(3, L.FEAT_SYNC_DEV)], unbounded_thr=400.0, precision=precision,
                       keep_final=False, keep_steps=True, csr_row=torch.tensor(csr[0], device=device),
                       csr_col=torch.tensor(csr[1], device=device))
    return solve(req)


def rossler_labels(features: torch.Tensor, status: torch.Tensor) -> torch.Tensor:
    """0 synchronised (max deviation < 1.5), 1 not, 2 unbounded."""
    from pybasin_b200 import _lib as L

    lab = torch.where(features[:, 0] < 1.5, 0, 1)
    return torch.where(status == L.TRAJ_UNBOUNDED, 2, lab).to(torch.int32)


def per_point_fractions(labels: torch.Tensor, group: torch.Tensor, n_points: int, n_classes: int) -> torch.Tensor:
    """(P, C) class fractions of each parameter point."""
    idx = group.to(torch.int64) * n_classes + labels.to(torch.int64)
    c = torch.bincount(idx, minlength=n_points * n_classes).view(n_points, n_classes).double()
    return c / c.sum(dim=1, keepdim=True).clamp_min(1)
