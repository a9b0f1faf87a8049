"""Surrogate-gated basin-stability pass.

ICs -> surrogate logits -> confidence gate (threshold, seeded audit slice) ->
the routed ICs (low confidence or audited) are integrated with the fused Dopri5
pipeline together with the templates -> labels merged back -> counts.  Every
label is either an integrator label or a confident surrogate label, and the
audit slice measures how often a confident surrogate label disagrees with the
integrator; where that happens too often at a parameter point (or over the whole
pass), the point's surrogate labels are replaced by integrated ones.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from pybasin_b200 import _lib as L
from pybasin_b200.pipeline import BasinStabilityPipeline, to_host_pinned
from pybasin_b200.surrogate import MLPSurrogate, TrainHistory, _bind, _p
from pybasin_b200.train import GraphTrainer


class GateStats:
    """Gate statistics of one pass; the audit tally stays on the device until read."""

    def __init__(self, n: int, n_routed: int, tally: torch.Tensor | None):
        self.n = n
        self.n_routed = n_routed
        self.n_fallback = 0  # ICs of points whose audit failed, integrated as well
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
    def integrated_fraction(self) -> float:
        """Routed by the gate or by a failed audit: labelled by the integrator."""
        return (self.n_routed + self.n_fallback) / max(self.n, 1)


def calibrate_temperature_device(logits: torch.Tensor, labels: torch.Tensor, lo: float = 0.5, hi: float = 4.0,
                                 steps: int = 71) -> torch.Tensor:
    """The temperature of :func:`calibrate_temperature`, computed on the device
    (a 0-d tensor; nothing waits for it): the grid point over [lo, hi] minimising the
    mean negative log-likelihood of ``labels`` under ``logits / T``."""
    grid = torch.linspace(lo, hi, steps, device=logits.device, dtype=torch.float64)
    z = logits.to(torch.float64)[None] / grid[:, None, None]
    lab = labels.to(torch.int64)
    nll = torch.logsumexp(z, dim=2) - z.gather(2, lab[None, :, None].expand(steps, -1, 1))[..., 0]
    return grid[torch.argmin(nll.mean(dim=1))].to(torch.float32)


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


class FitInfo:
    """What one :meth:`SurrogateGatedPipeline.fit` did; reading it waits for the device."""

    def __init__(self, trainers: list, n_train: int, n_calibration: int, owner: "SurrogateGatedPipeline"):
        self.trainers = trainers
        self.n_train = n_train
        self.n_calibration = n_calibration
        self._owner = owner

    @property
    def temperature(self) -> float:
        T = getattr(self._owner, "_temperature_dev", None)
        return 1.0 if T is None else float(T.item())

    def summary(self) -> dict:
        st = [t.stats() for t in self.trainers]
        return {"n_train": self.n_train, "n_calibration": self.n_calibration, "temperature": self.temperature,
                "train_accuracy": st[-1]["accuracy"], "train_error_flag": max(x["error"] for x in st),
                "train_steps": sum(t.steps for t in self.trainers),
                "train_launches": sum(t.launches for t in self.trainers),
                "train_flop": sum(t.flops() for t in self.trainers),
                "graph_capture_s": sum(t.capture_s for t in self.trainers)}


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
        max_chunk: int = 1 << 20,
        audit_tolerance: float | None = 0.002,
        audit_min_disagree: int = 3,
    ):
        self.pipe = pipeline
        self.max_chunk = max_chunk
        self.audit_tolerance = audit_tolerance
        self.audit_min_disagree = audit_min_disagree
        self.dev = pipeline.dev
        # the parameter points (a study's rows; the pipeline's last row is the templates')
        self.n_groups = pipeline.n_groups
        self.param_table = pipeline.params[: self.n_groups].to(torch.float64).contiguous()
        self.params = self.param_table[0]  # the main parameter row
        self.S = pipeline.dim
        self.C = pipeline.n_classes + 1  # + unbounded
        self.net = MLPSurrogate(self.S + self.params.numel(), self.C, hidden=hidden, depth=depth, seed=seed,
                                device=self.dev, n_freq=n_freq, freq_scale=freq_scale, pad_inputs=True)
        self._trainers: dict[tuple, GraphTrainer] = {}
        self.calib_fraction = calib_fraction
        self.temperature = 1.0
        self.threshold = threshold
        self.audit_fraction = audit_fraction
        self.audit_seed = audit_seed
        self._audit: dict[int, torch.Tensor] = {}

    # -- training ------------------------------------------------------------------
    def _raw_inputs(self, y0: torch.Tensor, group: torch.Tensor | None = None) -> torch.Tensor:
        if group is None:
            p = self.params.to(torch.float32).expand(y0.shape[0], -1)
        else:
            p = self.param_table.to(torch.float32).index_select(0, group.to(self.dev, torch.int64))
        return torch.cat([y0.to(torch.float32), p], dim=1)

    def _x(self, y0: torch.Tensor, group: torch.Tensor | None = None) -> torch.Tensor:
        """Network inputs of ICs (with the parameter point of each for a study)."""
        if group is None:
            return self.net.inputs(y0, self.params)
        return self.net.inputs(y0, self.param_table, group)

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

    def _trainer(self, n_rows: int, epochs: int, batch: int, lr: float, resume: bool, seed: int) -> GraphTrainer:
        key = (n_rows, epochs, batch, lr, resume, seed)
        tr = self._trainers.get(key)
        if tr is None:
            tr = GraphTrainer(self.net, n_rows=n_rows, epochs=epochs, batch=batch, lr=lr, seed=seed, resume=resume)
            self._trainers[key] = tr
        return tr

    def fit(self, y0_random: torch.Tensor, y0_pool: torch.Tensor | None = None, n_active: int = 0,
            epochs: int = 40, batch: int = 4096, lr: float = 5e-3, seed: int = 0,
            group_random: torch.Tensor | None = None, group_pool: torch.Tensor | None = None) -> "FitInfo":
        """Train the surrogate on labels of the integrator, on the tensor cores
        (``GraphTrainer``: one captured CUDA graph per training run), without a host
        round trip: every step is queued on the current stream.

        The first ``calib_fraction`` of ``y0_random`` (device ICs) is held out for
        calibration, the rest is labelled by the integrator and trained on.  With
        ``n_active`` > 0 that first run takes ``epochs // 2`` epochs; then the
        ``n_active`` ICs of ``y0_pool`` the network is least confident about
        (labels where the basins interleave) are labelled too, and training resumes
        on both sets for ``epochs`` epochs.  Last, the softmax temperature minimising
        the held-out negative log-likelihood is folded into the last layer, so the
        gate's threshold reads as a probability of the label being right.  For a
        parameter study, ``group_random`` / ``group_pool`` give each IC's point: the
        network then sees the point's parameters next to the IC."""
        lib = L.load()
        _bind(lib)
        s = torch.cuda.current_stream(self.dev).cuda_stream
        net = self.net
        n = y0_random.shape[0]
        n_cal = int(n * self.calib_fraction) if n >= 100 else 0
        g_r = None if group_random is None else group_random.to(self.dev, torch.int32)
        labels, _ = self.pipe.run_device(y0_random, group=g_r)
        lab = labels.clone()
        fit_ic, fit_lab = y0_random[n_cal:], lab[n_cal:]
        g_fit = None if g_r is None else g_r[n_cal:]
        net.fit_normalisation(self._raw_inputs(fit_ic, g_fit))
        x_r = self._x(fit_ic, g_fit)
        active = n_active > 0 and y0_pool is not None
        tr1 = self._trainer(n - n_cal, max(epochs // 2, 1) if active else epochs, batch, lr, False, seed)
        tr1.train(x_r, fit_lab)
        trainers = [tr1]
        if active:
            m = y0_pool.shape[0]
            g_p = None if group_pool is None else group_pool.to(self.dev, torch.int32)
            logits = net.logits(self._x(y0_pool, g_p))
            label = torch.empty((m,), dtype=torch.int32, device=self.dev)
            conf = torch.empty((m,), dtype=torch.float32, device=self.dev)
            route = torch.empty((m,), dtype=torch.int32, device=self.dev)
            n_route = torch.empty((1,), dtype=torch.int32, device=self.dev)
            # threshold 0: nothing routed, only the confidences wanted
            L.check(lib.pb_surrogate_gate(_p(logits), m, self.C, 0.0, None, _p(label), _p(conf), _p(route),
                                          _p(n_route), s), "pb_surrogate_gate")
            pick = torch.topk(conf, min(n_active, m), largest=False).indices
            y0_act = y0_pool.index_select(0, pick).contiguous()
            g_a = None if g_p is None else g_p.index_select(0, pick).contiguous()
            lab_a, _ = self.pipe.run_device(y0_act, group=g_a)
            x_all = torch.cat([x_r, self._x(y0_act, g_a)])
            lab_all = torch.cat([fit_lab, lab_a])
            tr2 = self._trainer(x_all.shape[0], epochs, batch, lr, True, seed + 1)
            tr2.train(x_all, lab_all)
            trainers.append(tr2)
        if n_cal > 0:
            z = net.logits(self._x(y0_random[:n_cal], None if g_r is None else g_r[:n_cal]))
            T = calibrate_temperature_device(z, lab[:n_cal])
            net.W[-1].div_(T)
            net.b[-1].div_(T)
            net.Wb[-1].copy_(net.W[-1])
            net._step += 1  # repack the inference weights
            self._temperature_dev = T
        return FitInfo(trainers, n - n_cal + (n_active if active else 0), n_cal, self)

    # -- inference -------------------------------------------------------------------
    def audit_mask(self, n: int) -> torch.Tensor:
        m = self._audit.get(n)
        if m is None:
            rng = np.random.default_rng(self.audit_seed)
            m = torch.as_tensor((rng.random(n) < self.audit_fraction).astype(np.uint8), device=self.dev)
            self._audit[n] = m
        return m

    def run_device(self, y0: torch.Tensor, group: torch.Tensor | None = None
                   ) -> tuple[torch.Tensor, torch.Tensor, GateStats]:
        """Labels (int32, class n_classes = unbounded) and per-class counts for device
        ICs; for a parameter study ``group`` gives each IC's point and the counts are
        per point, (points, classes)."""
        lib = L.load()
        _bind(lib)
        s = torch.cuda.current_stream(self.dev).cuda_stream
        n = y0.shape[0]
        grp = None if group is None else group.to(self.dev, torch.int32).contiguous()
        x = self._x(y0, grp)
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
            # integrated in chunks of at most max_chunk ICs: the deferred dense output's
            # step records are sized per trajectory (1024 records of 48 B for one FP32
            # state), so a chunk bounds the scratch (1M ICs: 48 GiB)
            routed_g = None
            if grp is not None:  # the routed ICs' points (int32 moved as 4-byte words)
                routed_g = torch.empty((k,), dtype=torch.int32, device=self.dev)
                L.check(lib.pb_gather_rows(_p(grp), 1, _p(route), _p(n_route), k, _p(routed_g), s),
                        "pb_gather_rows")
            if k <= self.max_chunk:
                integ, _ = self.pipe.run_device(routed, group=routed_g)
            else:
                integ = torch.empty((k,), dtype=torch.int32, device=self.dev)
                for c0 in range(0, k, self.max_chunk):
                    c1 = min(k, c0 + self.max_chunk)
                    lab_c, _ = self.pipe.run_device(routed[c0:c1], group=None if routed_g is None else routed_g[c0:c1])
                    integ[c0:c1].copy_(lab_c)
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
        n_fallback = 0
        if k > 0 and self.audit_tolerance is not None:
            n_fallback = self._audit_fallback(y0, grp, label, route[:k], sur_of_routed, integ, conf, audit)
            if n_fallback > 0 and grp is None:
                counts.copy_(torch.bincount(label.to(torch.int64), minlength=self.C))
        if grp is not None:  # per point: (points, classes)
            idx = grp.to(torch.int64) * self.C + label.to(torch.int64)
            counts = torch.bincount(idx, minlength=self.n_groups * self.C).view(self.n_groups, self.C)
        st = GateStats(n, k, tally)
        st.n_fallback = n_fallback
        return label, counts, st

    def _audit_fallback(self, y0, grp, label, route, sur_of_routed, integ, conf, audit) -> int:
        """The audit judges the surrogate point by point: where the audited confident
        labels of a parameter point (of the whole pass without a study) disagree with
        the integrator's in more than ``audit_tolerance`` of them (and at least
        ``audit_min_disagree`` times), every IC of that point the surrogate labelled
        is integrated too and takes the integrator's label.  Returns how many."""
        P = self.n_groups if grp is not None else 1
        n = y0.shape[0]
        r = route.to(torch.int64)
        g_all = grp.to(torch.int64) if grp is not None else torch.zeros((n,), dtype=torch.int64, device=self.dev)
        g_r = g_all.index_select(0, r)
        aud = audit.index_select(0, r).bool() & (conf.index_select(0, r) >= self.threshold)
        dis = aud & (sur_of_routed != integ)
        n_aud = torch.bincount(g_r[aud], minlength=P).double()
        n_dis = torch.bincount(g_r[dis], minlength=P).double()
        bad = (n_dis >= self.audit_min_disagree) & (n_dis > self.audit_tolerance * n_aud)
        self.last_fallback_points = bad
        if not bool(bad.any()):  # one host read
            return 0
        routed = torch.zeros((n,), dtype=torch.bool, device=self.dev)
        routed[r] = True
        extra = torch.nonzero(bad.index_select(0, g_all) & ~routed).flatten()
        m = extra.numel()
        if m == 0:
            return 0
        ye = y0.index_select(0, extra).contiguous()
        ge = None if grp is None else grp.index_select(0, extra).contiguous()
        for c0 in range(0, m, self.max_chunk):
            c1 = min(m, c0 + self.max_chunk)
            lab_c, _ = self.pipe.run_device(ye[c0:c1], group=None if ge is None else ge[c0:c1])
            label[extra[c0:c1]] = lab_c
        return m

    def run(self, y0_host: torch.Tensor, names: bool = True, group: torch.Tensor | None = None):
        """Host ICs -> (labels, basin stability per class, gate statistics); labels as
        class names, or with ``names=False`` as int32 indices into
        ``pipe.classes + ["unbounded"]`` (no per-IC string objects to build).  For a
        parameter study (``group``: each IC's point) the basin stability is a list
        with one dict per point."""
        with torch.cuda.device(self.dev):
            y0 = y0_host.to(self.dev, dtype=torch.float32, non_blocking=True)
            g = None if group is None else group.to(self.dev, dtype=torch.int32, non_blocking=True)
            label, counts, stats = self.run_device(y0, g)
            lab, cnt = to_host_pinned(self, label, counts)
        classes = np.array(self.pipe.classes + ["unbounded"], dtype=object)

        def fractions(c):
            n = max(int(c.sum()), 1)
            return {classes[i]: float(c[i]) / n for i in range(len(classes)) if c[i] > 0}

        bs = fractions(cnt) if group is None else [fractions(row) for row in cnt.reshape(self.n_groups, self.C)]
        return (classes[lab] if names else lab.copy()), bs, stats
