"""Surrogate-gated basin-stability pass.

ICs -> surrogate logits -> confidence gate (threshold, seeded audit slice) ->
the routed ICs (low confidence or audited) are integrated with the fused Dopri5
pipeline together with the templates -> labels merged back -> counts.  Every
label is either an integrator label or a confident surrogate label, and the
audit slice measures how often a confident surrogate label disagrees with the
integrator.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from pybasin_b200 import _lib as L
from pybasin_b200.pipeline import BasinStabilityPipeline, to_host_pinned
from pybasin_b200.surrogate import MLPSurrogate, TrainHistory, _bind, _p


class GateStats:
    """Gate statistics of one pass; the audit tally stays on the device until read."""

    def __init__(self, n: int, n_routed: int, tally: torch.Tensor | None):
        self.n = n
        self.n_routed = n_routed
        self._tally = tally  # int32 (3,): audited, audited-and-confident, ... of which relabelled
        self._host: list[int] | None = None

    def _read(self) -> list[int]:
        if self._host is None:
            self._host = [0, 0, 0] if self._tally is None else [int(v) for v in self._tally.cpu().tolist()]
        return self._host

    @property
    def n_audited(self) -> int:
        return self._read()[0]

    @property
    def audit_confident(self) -> int:
        """Audited rows the surrogate was confident about."""
        return self._read()[1]

    @property
    def audit_disagree(self) -> int:
        """... of which the integrator gave another label."""
        return self._read()[2]

    @property
    def routed_fraction(self) -> float:
        return self.n_routed / max(self.n, 1)

    @property
    def audit_error(self) -> float:
        return self.audit_disagree / max(self.audit_confident, 1)

    @property
    def routed_fraction(self) -> float:
        return self.n_routed / max(self.n, 1)

    @property
    def audit_error(self) -> float:
        return self.audit_disagree / max(self.audit_confident, 1)


def calibrate_temperature(logits: np.ndarray, labels: np.ndarray, grid: np.ndarray | None = None) -> float:
    """Softmax temperature minimising the mean negative log-likelihood of ``labels``
    under ``logits / T`` (a grid over [0.5, 4])."""
    grid = np.linspace(0.5, 4.0, 71) if grid is None else grid
    lab = labels.astype(np.int64)
    best_t, best_nll = 1.0, np.inf
    for T in grid:
        z = logits / T
        z = z - z.max(axis=1, keepdims=True)
        nll = float(np.mean(np.log(np.exp(z).sum(axis=1)) - z[np.arange(len(lab)), lab]))
        if nll < best_nll:
            best_t, best_nll = float(T), nll
    return best_t


class SurrogateGatedPipeline:
    """Surrogate in front of a ``BasinStabilityPipeline`` for one ODE system and parameter row."""

    def __init__(
        self,
        pipeline: BasinStabilityPipeline,
        hidden: int = 256,
        depth: int = 4,
        threshold: float = 0.95,
        audit_fraction: float = 0.01,
        audit_seed: int = 123,
        seed: int = 0,
        n_freq: int = 64,
        freq_scale: float = 0.3,
        calib_fraction: float = 0.1,
    ):
        self.pipe = pipeline
        self.dev = pipeline.dev
        self.params = pipeline.params[0].to(torch.float64)  # the main parameter row
        self.S = pipeline.dim
        self.C = pipeline.n_classes + 1  # + unbounded
        self.net = MLPSurrogate(self.S + self.params.numel(), self.C, hidden=hidden, depth=depth, seed=seed,
                                device=self.dev, n_freq=n_freq, freq_scale=freq_scale)
        self.calib_fraction = calib_fraction
        self.temperature = 1.0
        self.threshold = threshold
        self.audit_fraction = audit_fraction
        self.audit_seed = audit_seed
        self._audit: dict[int, torch.Tensor] = {}

    # -- training ------------------------------------------------------------------
    def _raw_inputs(self, y0: torch.Tensor) -> torch.Tensor:
        p = self.params.to(torch.float32).expand(y0.shape[0], -1)
        return torch.cat([y0.to(torch.float32), p], dim=1)

    def train(self, y0_train: torch.Tensor, epochs: int = 30, batch: int = 1024, lr: float = 2e-3,
              seed: int = 0) -> tuple[TrainHistory, dict[str, float]]:
        """Label ``y0_train`` with the integrator, fit the network on all but a
        ``calib_fraction`` slice of those labels, then calibrate its confidence on
        the held-out slice: the softmax temperature T minimising the held-out
        negative log-likelihood, folded into the last layer, so that the gate's
        threshold reads as a probability of the label being right."""
        t0 = time.perf_counter()
        y0_train = y0_train.to(self.dev)
        labels, _ = self.pipe.run_device(y0_train)
        labels = labels.clone()
        torch.cuda.synchronize(self.dev)
        t1 = time.perf_counter()
        n = y0_train.shape[0]
        n_cal = int(n * self.calib_fraction) if n >= 100 else 0
        fit_ic, fit_lab = y0_train[n_cal:], labels[n_cal:]
        self.net.fit_normalisation(self._raw_inputs(fit_ic))
        x = self.net.inputs(fit_ic, self.params)
        hist = self.net.train(x, fit_lab, epochs=epochs, batch=batch, lr=lr, seed=seed)
        if n_cal > 0:
            z = self.net.logits(self.net.inputs(y0_train[:n_cal], self.params)).double().cpu().numpy()
            self.temperature = calibrate_temperature(z, labels[:n_cal].cpu().numpy())
            self.net.fold_temperature(self.temperature)
        torch.cuda.synchronize(self.dev)
        t2 = time.perf_counter()
        return hist, {"label_s": t1 - t0, "train_s": t2 - t1, "n_train": int(n - n_cal), "n_calibration": n_cal,
                      "temperature": self.temperature}

    # -- inference -------------------------------------------------------------------
    def audit_mask(self, n: int) -> torch.Tensor:
        m = self._audit.get(n)
        if m is None:
            rng = np.random.default_rng(self.audit_seed)
            m = torch.as_tensor((rng.random(n) < self.audit_fraction).astype(np.uint8), device=self.dev)
            self._audit[n] = m
        return m

    def run_device(self, y0: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor, GateStats]:
        """Labels (int32, class n_classes = unbounded) and per-class counts for device ICs."""
        lib = L.load()
        _bind(lib)
        s = torch.cuda.current_stream(self.dev).cuda_stream
        n = y0.shape[0]
        x = self.net.inputs(y0, self.params)
        logits = self.net.logits(x)
        audit = self.audit_mask(n)
        label = torch.empty((n,), dtype=torch.int32, device=self.dev)
        route = torch.empty((n,), dtype=torch.int32, device=self.dev)
        n_route = torch.empty((1,), dtype=torch.int32, device=self.dev)
        conf = torch.empty((n,), dtype=torch.float32, device=self.dev)
        L.check(lib.pb_surrogate_gate(_p(logits), n, self.C, self.threshold, _p(audit), _p(label), _p(conf),
                                      _p(route), _p(n_route), s), "pb_surrogate_gate")
        k = int(n_route.item())  # the one host read of the pass: how many ICs to integrate
        if k > 0:
            routed = torch.empty((k, self.S), dtype=torch.float32, device=self.dev)
            L.check(lib.pb_gather_rows(_p(y0.contiguous()), self.S, _p(route), _p(n_route), k, _p(routed), s),
                    "pb_gather_rows")
            integ, _ = self.pipe.run_device(routed)
            sur_of_routed = torch.empty((k,), dtype=torch.int32, device=self.dev)
            L.check(lib.pb_merge_labels(_p(integ), _p(route), _p(n_route), k, _p(label), _p(sur_of_routed), s),
                    "pb_merge_labels")
        else:
            integ = sur_of_routed = None
        counts = torch.empty((self.C,), dtype=torch.int64, device=self.dev)
        tally = torch.empty((3,), dtype=torch.int32, device=self.dev)
        L.check(lib.pb_gate_summary(_p(label), n, self.C, _p(route) if k > 0 else None, _p(n_route), k, _p(audit),
                                    _p(conf), self.threshold, _p(sur_of_routed), _p(integ), _p(counts), _p(tally), s),
                "pb_gate_summary")
        return label, counts, GateStats(n, k, tally)

    def run(self, y0_host: torch.Tensor, names: bool = True) -> tuple[np.ndarray, dict[str, float], GateStats]:
        """Host ICs -> (labels, basin stability per class, gate statistics); labels as
        class names, or with ``names=False`` as int32 indices into
        ``pipe.classes + ["unbounded"]`` (no per-IC string objects to build)."""
        with torch.cuda.device(self.dev):
            y0 = y0_host.to(self.dev, dtype=torch.float32, non_blocking=True)
            label, counts, stats = self.run_device(y0)
            lab, cnt = to_host_pinned(self, label, counts)
        classes = np.array(self.pipe.classes + ["unbounded"], dtype=object)
        n = max(int(cnt.sum()), 1)
        bs = {classes[i]: float(cnt[i]) / n for i in range(len(classes)) if cnt[i] > 0}
        return (classes[lab] if names else lab.copy()), bs, stats
