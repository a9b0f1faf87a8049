"""``B200Dopri5Solver``: the drop-in for the reference's ``TorchDiffEqSolver``.

It satisfies the reference's ``SolverProtocol`` (src/pybasin/protocols.py:116-187):
``device``, the constructor arguments (``t_span, t_steps, device, method, rtol,
atol, cache_dir, t_eval``), ``integrate(ode_system, y0, params=None) -> (t, y)``
and ``clone(*, device, t_steps_factor, cache_dir)``, with the base class's
argument checks and IC-major parameter expansion
(src/pybasin/solvers/base.py:36-183).  Integration is the per-trajectory
Dopri5 kernel of the CUDA library; there is no CPU path.

Two output modes:

* ``output="full"`` returns ``y`` of shape ``(t_steps, B*P, S)`` exactly like the
  reference solvers, so any reference feature extractor works on it.
* ``output="fused"`` (the default when a ``FusedFeatureExtractor`` is given)
  keeps no trajectory: the window statistics are computed inside the kernel,
  ``y`` is the state at the end of the span with shape ``(1, B*P, S)``, and the
  features ride on ``y`` for ``FusedFeatureExtractor.extract_features``.
  Trajectories stopped by the unbounded event get ``inf`` rows (the diffrax
  convention the reference relies on, basin_stability_estimator.py:519-527).
"""

from __future__ import annotations

import logging
import threading
from dataclasses import dataclass
from typing import Any

import numpy as np
import torch

from pybasin_b200 import _lib as L
from pybasin_b200.engine import FeatureColumn, MortonOrder, SolveRequest, solve
from pybasin_b200.features import FusedFeatureExtractor
from pybasin_b200.odes import resolve_system

logger = logging.getLogger(__name__)

_UNSET = object()

#: reference default max_steps of the per-trajectory solvers (jax_solver.py:37)
DEFAULT_MAX_STEPS = 16**5

#: tolerance floor of the FP32-stage kernel: rtol below FP32 resolution makes the
#: embedded error estimate pure rounding noise (the reference's own docs warn of
#: stagnation, docs/user-guide/solvers.md:206-211)
MIXED_RTOL_FLOOR = 1e-6


class IntegrationResult(tuple):
    """``(t, y)`` that also carries ``features``, ``feature_names`` and ``status``."""

    features: torch.Tensor | None
    feature_names: list[str]
    status: torch.Tensor
    steps: torch.Tensor | None

    def __new__(cls, t: torch.Tensor, y: torch.Tensor, **extra: Any) -> "IntegrationResult":
        obj = super().__new__(cls, (t, y))
        for k, v in extra.items():
            setattr(obj, k, v)
        return obj


@dataclass
class OrbitData:
    """Field layout of the reference's ``OrbitData`` (src/pybasin/utils.py:228-251):
    ``peak_values`` (max_peaks, B, D) NaN-padded, ``peak_counts`` (B, D)."""

    peak_values: torch.Tensor
    peak_counts: torch.Tensor
    dof_indices: list[int]
    time_steady: float


class _OrbitColumns:
    """Feature columns of an orbit-data solve: one peak count per state in ``dof``."""

    def __init__(self, dof: list[int], support: int, time_steady: float | None):
        self.dof, self.support, self.time_steady = dof, int(support), time_steady
        self.resolved = 0.0
        if self.support < 1:
            raise ValueError("peak_support must be >= 1")

    def columns(self, num_states: int) -> list[FeatureColumn]:
        if any(not 0 <= d < num_states for d in self.dof):
            raise ValueError(f"dof indices must lie in [0, {num_states})")
        return [FeatureColumn(d, L.FEAT_NUMBER_PEAKS, float(self.support), f"state_{d}__peaks") for d in self.dof]

    def resolve_time_steady(self, save_ts: torch.Tensor) -> float:
        if self.time_steady is not None:
            self.resolved = float(self.time_steady)
        else:
            t0, t1 = float(save_ts[0]), float(save_ts[-1])
            self.resolved = t0 + 0.85 * (t1 - t0)  # DEFAULT_STEADY_FRACTION, src/pybasin/constants.py
        return self.resolved


_streams = threading.local()


def _thread_stream(dev: torch.device) -> torch.cuda.Stream:
    """One non-default stream per (host thread, device): concurrent integrate
    calls from the estimator's thread pool overlap on the GPU."""
    cache = getattr(_streams, "by_dev", None)
    if cache is None:
        cache = {}
        _streams.by_dev = cache
    s = cache.get(dev.index)
    if s is None:
        s = torch.cuda.Stream(device=dev)
        cache[dev.index] = s
    return s


class B200Dopri5Solver:
    """Adaptive Dormand-Prince 5(4) over many ICs on one B200, fused with features.

    :param t_span: integration interval ``(t0, t1)``.
    :param t_steps: number of save points in the save region.
    :param device: device of the returned tensors ('cuda', 'cuda:N', 'cpu' or None).
        Computation always runs on a CUDA device (``device`` if it is CUDA, else the
        current CUDA device); a CPU ``device`` only means CPU output tensors, which is
        what the reference's TemplateIntegrator asks for (template_integrator.py:80-86).
    :param method: only ``"dopri5"``.
    :param rtol: relative tolerance (the FP32-stage kernel uses ``max(rtol, mixed_rtol_floor)``).
    :param atol: absolute tolerance.
    :param cache_dir: directory of the result cache (``None`` = no cache).  A result is
        stored as ``{t, y, features, status}`` in a safetensors file keyed by an MD5
        of the system, its parameters, the ICs, the save grid and every setting that
        changes the result (the reference's CacheManager key,
        src/pybasin/cache_manager.py:27-68, here with the fused features and statuses
        instead of the full trajectory in fused mode).
    :param t_eval: save region ``(save_start, save_end)`` within ``t_span``.
    :param precision: ``"fp64"`` (plain FP64 kernel) or ``"mixed"`` (FP32 stages and
        state, FP64 time, error norm and step control).
    :param feature_extractor: a ``FusedFeatureExtractor`` whose statistics the kernel computes.
    :param output: ``"fused"`` or ``"full"`` (default: fused iff a feature extractor is given).
    :param max_steps: attempted steps per trajectory before giving up (status MAX_STEPS).
    :param unbounded_threshold: stop a trajectory once max|y| >= this after an accepted
        step (the reference's stop events, e.g. case_studies/lorenz/setup_lorenz_system.py:16-26).
    :param schedule: ``"queue"`` (persistent warps + work queue), ``"probed"`` (the queue in
        predicted-cost order: a probe over the first 5 % of the span orders the
        trajectories longest first; identical results) or ``"plain"``.
    :param dense_mode: ``"deferred"`` (the integrator writes one record per window step that
        holds save points and a warp-parallel pass evaluates the save points) or ``"inline"``
        (each thread evaluates its save points after its step); full output is always inline.
    :param order: ``"morton"`` integrates the ICs in Z-order of their coordinates so each
        warp holds neighbouring ICs (similar dynamics and step counts); ``"none"`` keeps
        the input order.  Outputs are in input order either way.
    """

    def __init__(
        self,
        t_span: tuple[float, float] = (0, 1000),
        t_steps: int = 1000,
        device: str | None = None,
        method: str = "dopri5",
        rtol: float = 1e-8,
        atol: float = 1e-6,
        cache_dir: str | None = None,
        t_eval: tuple[float, float] | None = None,
        *,
        precision: str = "fp64",
        feature_extractor: FusedFeatureExtractor | None = None,
        output: str | None = None,
        max_steps: int = DEFAULT_MAX_STEPS,
        unbounded_threshold: float | None = None,
        schedule: str = "probed",
        mixed_rtol_floor: float = MIXED_RTOL_FLOOR,
        block_size: int = 0,
        grid_blocks: int = 0,
        order: str = "morton",
        dense_mode: str = "deferred",
        refill_lanes: int = 0,
    ):
        if t_eval is not None and (t_eval[0] < t_span[0] or t_eval[1] > t_span[1]):
            raise ValueError(f"t_eval {t_eval} must be within t_span {t_span}.")
        if method not in ("dopri5", None):
            raise ValueError(f"B200Dopri5Solver implements method='dopri5' only, got {method!r}")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if output not in (None, "fused", "full"):
            raise ValueError("output must be 'fused' or 'full'")
        if schedule not in L.SCHEDULES:
            raise ValueError(f"schedule must be one of {sorted(L.SCHEDULES)}")
        if t_steps < 1:
            raise ValueError("t_steps must be >= 1")
        if order not in ("morton", "none"):
            raise ValueError("order must be 'morton' or 'none'")
        if dense_mode not in ("deferred", "inline"):
            raise ValueError("dense_mode must be 'deferred' or 'inline'")
        if not 0 <= refill_lanes <= 32:
            raise ValueError("refill_lanes must be in [0, 32] (0 or 32: refill only a fully idle warp)")
        self.refill_lanes = int(refill_lanes)
        self.order = order
        self.dense_mode = dense_mode
        self.t_span = t_span
        self.t_eval = t_eval
        self.t_steps = t_steps
        self.method = "dopri5"
        self.rtol = rtol
        self.atol = atol
        self.precision = precision
        self.feature_extractor = feature_extractor
        self.output = output or ("fused" if feature_extractor is not None else "full")
        if self.output == "fused" and feature_extractor is None:
            raise ValueError("output='fused' needs a FusedFeatureExtractor")
        self.max_steps = int(max_steps)
        self.unbounded_threshold = unbounded_threshold
        self.schedule = schedule
        self.mixed_rtol_floor = mixed_rtol_floor
        self.block_size = block_size
        self.grid_blocks = grid_blocks
        self._cache_dir = cache_dir
        self._set_device(device)

    # -- reference Solver surface ---------------------------------------------
    def _set_device(self, device: str | None) -> None:
        # same normalisation as src/pybasin/solvers/base.py:73-97
        self._device_str = device
        if device is None:
            self.device = torch.device("cuda:0" if torch.cuda.is_available() else "cpu")
        else:
            dev = torch.device(device)
            if dev.type == "cuda":
                self.device = torch.device(f"cuda:{dev.index if dev.index is not None else 0}")
            else:
                self.device = dev

    def clone(
        self,
        *,
        device: str | None = None,
        t_steps_factor: int = 1,
        cache_dir: str | None | object = _UNSET,
    ) -> "B200Dopri5Solver":
        """Copy with a new output device / resolution (protocols.py:170-187)."""
        return B200Dopri5Solver(
            t_span=self.t_span,
            t_steps=self.t_steps * t_steps_factor,
            device=device or self._device_str,
            method=self.method,
            rtol=self.rtol,
            atol=self.atol,
            cache_dir=self._cache_dir if cache_dir is _UNSET else cache_dir,  # type: ignore[arg-type]
            t_eval=self.t_eval,
            precision=self.precision,
            feature_extractor=self.feature_extractor,
            output=self.output,
            max_steps=self.max_steps,
            unbounded_threshold=self.unbounded_threshold,
            schedule=self.schedule,
            mixed_rtol_floor=self.mixed_rtol_floor,
            block_size=self.block_size,
            grid_blocks=self.grid_blocks,
            order=self.order,
            dense_mode=self.dense_mode,
            refill_lanes=self.refill_lanes,
        )

    def compute_device(self) -> torch.device:
        if not torch.cuda.is_available():
            raise RuntimeError("B200Dopri5Solver needs a CUDA device; there is no CPU fallback")
        if self.device.type == "cuda":
            return self.device
        return torch.device(f"cuda:{torch.cuda.current_device()}")

    def effective_tolerances(self) -> tuple[float, float]:
        if self.precision == "mixed":
            return max(self.rtol, self.mixed_rtol_floor), self.atol
        return self.rtol, self.atol

    def save_times(self, dtype: torch.dtype) -> torch.Tensor:
        """Save instants as the reference builds them: linspace in y0's dtype (base.py:113-127)."""
        s0, s1 = self.t_eval if self.t_eval is not None else self.t_span
        return torch.linspace(s0, s1, self.t_steps, dtype=dtype)

    def integrate(
        self, ode_system: Any, y0: torch.Tensor, params: torch.Tensor | None = None
    ) -> IntegrationResult:
        """Integrate every row of ``y0`` (against every row of ``params`` if given).

        Returns ``(t, y)``; ``y`` has shape ``(t_steps, B*P, S)`` in full mode and
        ``(1, B*P, S)`` in fused mode, trajectory ``ic*P + p`` carrying
        ``(y0[ic], params[p])`` (base.py:155-159).
        """
        if self._cache_dir is None:
            return self._integrate(ode_system, y0, params, self.feature_extractor, 0)
        from pybasin_b200 import result_cache

        return result_cache.cached_integrate(self, ode_system, y0, params)

    def orbit_data(
        self,
        ode_system: Any,
        y0: torch.Tensor,
        dof: list[int],
        time_steady: float | None = None,
        peak_support: int = 1,
        max_peaks: int = 256,
        params: torch.Tensor | None = None,
    ) -> "OrbitData":
        """Peak amplitudes of the steady-state window for orbit diagrams, computed in the
        solve (the reference's ``extract_orbit_data``, src/pybasin/utils.py:254-303:
        strict local maxima with ``peak_support`` neighbours on each side, for every
        state in ``dof``).  At most ``max_peaks`` values per trajectory and state are
        kept; ``peak_counts`` holds the full counts."""
        ext = _OrbitColumns(list(dof), peak_support, time_steady)
        r = self._integrate(ode_system, y0, params, ext, max_peaks)
        counts = r.features.to(torch.long)  # (B*P, D)
        keep = int(min(max(int(counts.max()) if counts.numel() else 0, 0), max_peaks))
        peaks = r.peaks[:, :, :keep].permute(2, 0, 1).contiguous()  # (max_peaks, B*P, D)
        return OrbitData(peaks, counts, list(dof), ext.resolved)

    def _integrate(self, ode_system: Any, y0: torch.Tensor, params: torch.Tensor | None, extractor: Any,
                   peak_cap: int) -> IntegrationResult:
        if y0.ndim != 2:
            raise ValueError(
                f"y0 must be 2D with shape (batch, n_dims), got shape {tuple(y0.shape)}. "
                f"For single initial condition, use y0.unsqueeze(0) or y0.reshape(1, -1)."
            )
        if y0.dtype not in (torch.float32, torch.float64):
            raise TypeError(f"y0 must be float32 or float64, got {y0.dtype}")
        B, S = y0.shape
        spec = resolve_system(ode_system, S)
        dev = self.compute_device()
        stream = _thread_stream(dev)
        save_host = self.save_times(y0.dtype)
        save_f64 = save_host.to(torch.float64)
        t0 = float(self.t_span[0])
        t1 = float(save_f64[-1])
        if params is not None:
            if params.ndim != 2:
                raise ValueError("params must be 2D with shape (P, n_params)")
            p_rows = params.detach().to(torch.float64).cpu().numpy()
            layout = L.LAYOUT_CROSS
        else:
            p_rows = spec.params[None, :]
            layout = L.LAYOUT_SINGLE
        P = p_rows.shape[0]
        n_traj = B * P if params is not None else B
        cols = extractor.columns(S) if extractor is not None else []
        if cols:
            ts = extractor.resolve_time_steady(save_host)
            idx = torch.nonzero(save_host >= ts)
            win_begin = int(idx[0, 0]) if idx.numel() > 0 else 0
        else:
            win_begin = 0
        rtol, atol = self.effective_tolerances()
        full = self.output == "full" and peak_cap == 0
        stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.device(dev), torch.cuda.stream(stream):
            y0_dev = y0.detach().to(dev, non_blocking=False).contiguous()
            params_dev = torch.as_tensor(np.ascontiguousarray(p_rows), device=dev)
            save_dev = save_f64.to(dev)
            order = None
            if self.order == "morton" and B > 1:
                ic_order = MortonOrder(dev)(y0_dev)
                if params is not None:
                    order = (ic_order.to(torch.int64)[:, None] * P + torch.arange(P, device=dev)).reshape(-1)
                    order = order.to(torch.int32)
                else:
                    order = ic_order
            csr_row = csr_col = None
            program = None
            if spec.system == L.SYS_USER:
                program = ode_system.program(L.PREC_MIXED if self.precision == "mixed" else L.PREC_FP64,
                                             dev.index if dev.index is not None else torch.cuda.current_device())
            if spec.system == L.SYS_ROSSLER_NET:
                from pybasin_b200.network import network_csr

                row, col, _ = network_csr(ode_system)
                csr_row = torch.as_tensor(row, dtype=torch.int32, device=dev)
                csr_col = torch.as_tensor(col, dtype=torch.int32, device=dev)
            req = SolveRequest(
                system=spec.system,
                dim=S,
                y0=y0_dev,
                params=params_dev,
                save_ts=save_dev,
                t_span=(t0, t1),
                rtol=rtol,
                atol=atol,
                layout=layout,
                n_traj=n_traj,
                win_begin=win_begin,
                columns=cols,
                precision=L.PREC_MIXED if self.precision == "mixed" else L.PREC_FP64,
                schedule=L.SCHEDULES[self.schedule],
                max_steps=self.max_steps,
                unbounded_thr=float(self.unbounded_threshold or 0.0),
                keep_final=not full,
                keep_full=full,
                out_dtype=y0.dtype,
                block_size=self.block_size,
                grid_blocks=self.grid_blocks,
                refill_lanes=self.refill_lanes,
                order=order,
                dense_mode=L.DENSE_DEFERRED if self.dense_mode == "deferred" else L.DENSE_INLINE,
                csr_row=csr_row,
                csr_col=csr_col,
                program=program,
                peak_cap=peak_cap,
            )
            res = solve(req, stream)
            if full:
                y = res.y_full
                t = save_host.to(self.device)
            else:
                y = res.y_final.unsqueeze(0)  # type: ignore[union-attr]
                t = save_host[-1:].to(self.device)
            status = res.status
            feats = res.features.to(y0.dtype) if res.features is not None else None
            if not full:
                unb = (status == L.TRAJ_UNBOUNDED).view(1, -1, 1)
                y = torch.where(unb, torch.full_like(y, float("inf")), y)
        stream.synchronize()
        y = y.to(self.device)  # type: ignore[union-attr]
        status = status.to(self.device)
        if feats is not None:
            feats = feats.to(self.device)
        names = [c.name for c in cols]
        if feats is None:
            feats = torch.zeros((n_traj, 0), dtype=y0.dtype, device=self.device)
        # side channel read by FusedFeatureExtractor.extract_features
        y._pb_features = feats  # type: ignore[attr-defined]
        y._pb_feature_names = names  # type: ignore[attr-defined]
        y._pb_status = status  # type: ignore[attr-defined]
        n_bad = int((status == L.TRAJ_MAX_STEPS).sum()) + int((status == L.TRAJ_NONFINITE).sum())
        if n_bad:
            logger.warning("B200Dopri5Solver: %d trajectories hit max_steps or went non-finite", n_bad)
        peaks = res.peaks.to(self.device) if res.peaks is not None else None
        return IntegrationResult(t, y, features=feats, feature_names=names, status=status, steps=None, peaks=peaks)
