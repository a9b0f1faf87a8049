"""GPU-resident basin-stability pass: ICs -> fused Dopri5 + features -> 1-NN labels -> counts.

This is the hot path of the reference's ``BasinStabilityEstimator.run`` for a
supervised 1-NN predictor (src/pybasin/basin_stability_estimator.py:230-361):
integration of the main and template ICs (:488-517), feature extraction
(:304-311), ``KNeighborsClassifier(n_neighbors=1)`` fit/predict (:426-446) and
the basin-stability fractions (:586-598).  Here the template ICs ride in the
same kernel launch as the main ICs (their own parameter row), the features never
leave the GPU, labelling is one kernel, and only labels and counts come back.

All buffers are allocated once per batch size so a pass can be captured into a
CUDA graph and replayed (``use_graph=True``).
"""

from __future__ import annotations

import ctypes
from typing import Any

import numpy as np
import torch

from pybasin_b200 import _lib as L
from pybasin_b200.engine import MortonOrder, SolveRequest, SolveResult, alloc_scratch, build_args, launch_solve
from pybasin_b200.odes import resolve_system
from pybasin_b200.solver import B200Dopri5Solver


def to_host_pinned(owner, label: torch.Tensor, counts: torch.Tensor) -> tuple[np.ndarray, np.ndarray]:
    """Labels and counts into page-locked host buffers kept on ``owner`` (grown as
    needed): two asynchronous copies and one stream synchronisation.  The arrays
    returned are views of those buffers, valid until the owner's next call."""
    n, c = label.numel(), counts.numel()
    buf = getattr(owner, "_host_out", None)
    if buf is None or buf[0].numel() < n or buf[1].numel() < c:
        buf = (torch.empty((max(n, 1),), dtype=label.dtype, pin_memory=True),
               torch.empty((max(c, 1),), dtype=counts.dtype, pin_memory=True))
        owner._host_out = buf
    hl, hc = buf[0][:n], buf[1][:c]
    hl.copy_(label.view(-1), non_blocking=True)
    hc.copy_(counts.view(-1), non_blocking=True)
    torch.cuda.current_stream(label.device).synchronize()
    return hl.numpy(), hc.numpy()


class BasinStabilityPipeline:
    """Labelled ICs for one ODE system and template set on one GPU.

    :param ode_system: reference-style ODE system (params mapping in TypedDict order).
    :param solver: a ``B200Dopri5Solver`` with a ``FusedFeatureExtractor`` (normalize=False).
    :param template_y0: template initial conditions (``TemplateIntegrator.template_y0``).
    :param template_labels: class name of each template.
    :param template_params: parameters for the templates (default: the system's).
    :param param_rows: parameter study: one row per parameter point, shape ``(P, n_params)``
        (default: the system's parameters, P = 1).  ICs pass their point through
        ``group`` in ``run_device``; counts come back per point.  As in the reference's
        parameter study, the templates are integrated once, at ``template_params``.
    """

    def __init__(
        self,
        ode_system: Any,
        solver: B200Dopri5Solver,
        template_y0: list[list[float]],
        template_labels: list[str],
        template_params: dict[str, float] | None = None,
        device: torch.device | str | None = None,
        param_rows: np.ndarray | None = None,
    ):
        fx = solver.feature_extractor
        if fx is None:
            raise ValueError("the pipeline needs a solver constructed with a FusedFeatureExtractor")
        if fx.normalize:
            raise ValueError("on-device 1-NN labelling uses raw features (FusedFeatureExtractor(normalize=False))")
        self.solver = solver
        self.dev = torch.device(device) if device is not None else solver.compute_device()
        self.dim = len(template_y0[0])
        self.spec = resolve_system(ode_system, self.dim)
        self.classes = sorted(set(template_labels), key=template_labels.index)
        self.n_classes = len(self.classes)
        self.tpl_class = torch.tensor(
            [self.classes.index(s) for s in template_labels], dtype=torch.int32, device=self.dev
        )
        tparams = (
            np.asarray(list(template_params.values()), dtype=np.float64)
            if template_params is not None
            else self.spec.params
        )
        rows = np.atleast_2d(np.asarray(param_rows, dtype=np.float64)) if param_rows is not None else self.spec.params[None]
        if rows.shape[1] != self.spec.params.shape[0]:
            raise ValueError(f"param_rows need {self.spec.params.shape[0]} columns")
        self.n_groups = rows.shape[0]
        # rows 0..P-1: parameter points; row P: the templates' parameters
        self.params = torch.tensor(np.vstack([rows, tparams[None]]), dtype=torch.float64, device=self.dev)
        self.ode_system = ode_system
        self.template_y0 = torch.tensor(template_y0, dtype=torch.float32, device=self.dev)
        self.morton = MortonOrder(self.dev)
        self.n_tpl = self.template_y0.shape[0]
        save = solver.save_times(torch.float32)
        self.save_ts = save.to(torch.float64).to(self.dev)
        self.columns = fx.columns(self.dim)
        ts = fx.resolve_time_steady(save)
        idx = torch.nonzero(save >= ts)
        self.win_begin = int(idx[0, 0]) if idx.numel() > 0 else 0
        self.t_span = (float(solver.t_span[0]), float(save[-1]))
        self._n: int | None = None
        self._graph: torch.cuda.CUDAGraph | None = None
        self.stream = torch.cuda.Stream(device=self.dev)

    # -- buffers ---------------------------------------------------------------
    def _allocate(self, capacity: int) -> None:
        """Buffers for up to `capacity` ICs; rows [n, n + templates) hold the templates."""
        dev = self.dev
        tot = capacity + self.n_tpl
        F = len(self.columns)
        self.capacity = capacity
        self.y0_buf = torch.empty((tot, self.dim), dtype=torch.float32, device=dev)
        self.pidx = torch.zeros((tot,), dtype=torch.int32, device=dev)
        self.out = SolveResult(
            features=torch.empty((tot, F), dtype=torch.float64, device=dev),
            status=torch.empty((tot,), dtype=torch.int32, device=dev),
            y_final=None,
            y_full=None,
            steps=torch.empty((tot,), dtype=torch.int64, device=dev),
        )
        self.queue = torch.zeros((1,), dtype=torch.int64, device=dev)
        self.order = torch.arange(tot, dtype=torch.int32, device=dev)
        self.labels = torch.empty((capacity,), dtype=torch.int32, device=dev)
        self.counts = torch.empty((self.n_groups, self.n_classes + 1), dtype=torch.int64, device=dev)
        rtol, atol = self.solver.effective_tolerances()
        req = SolveRequest(
            system=self.spec.system,
            dim=self.dim,
            y0=self.y0_buf,
            params=self.params,
            save_ts=self.save_ts,
            t_span=self.t_span,
            rtol=rtol,
            atol=atol,
            layout=L.LAYOUT_INDEXED,
            param_index=self.pidx,
            n_traj=tot,
            win_begin=self.win_begin,
            columns=self.columns,
            precision=L.PREC_MIXED if self.solver.precision == "mixed" else L.PREC_FP64,
            schedule=L.SCHEDULES[self.solver.schedule],
            max_steps=self.solver.max_steps,
            unbounded_thr=float(self.solver.unbounded_threshold or 0.0),
            keep_final=False,
            block_size=self.solver.block_size,
            grid_blocks=self.solver.grid_blocks,
            refill_lanes=getattr(self.solver, "refill_lanes", 0),
            order=self.order if self.solver.order == "morton" else None,
            dense_mode=L.DENSE_DEFERRED if self.solver.dense_mode == "deferred" else L.DENSE_INLINE,
        )
        self.program = None
        if self.spec.system == L.SYS_USER:
            prec = L.PREC_MIXED if self.solver.precision == "mixed" else L.PREC_FP64
            self.program = self.ode_system.program(prec, dev.index if dev.index is not None else None)
        self.args = build_args(req, self.out, self.queue, None)
        self.scratch = alloc_scratch(self.args, dev)  # sized for the full capacity
        self._n = None
        self._graph = None

    def release(self) -> None:
        """Drop the buffers sized for the largest batch so far (the next pass
        allocates again): the step-record scratch of 10^6 ICs is tens of GB."""
        for name in ("y0_buf", "pidx", "out", "queue", "order", "labels", "scratch", "args", "program"):
            if hasattr(self, name):
                delattr(self, name)
        self.capacity = -1
        self._n = None
        self._graph = None

    def _prepare(self, n: int, group: torch.Tensor | None = None) -> None:
        """Place the templates after the first n rows and size the launch to n + templates."""
        T = self.n_tpl
        self.y0_buf[n : n + T] = self.template_y0
        if group is None:
            self.pidx.zero_()
        else:
            self.pidx[:n].copy_(group.to(torch.int32), non_blocking=True)
        self.pidx[n : n + T] = self.n_groups
        if self.solver.order == "morton" and n > 1:
            grp = self.pidx[:n] if (group is not None and self.n_groups > 1) else None
            self.morton(self.y0_buf[:n], groups=grp, out=self.order[:n])
        elif self.solver.order == "morton":
            self.order[:n] = torch.arange(n, dtype=torch.int32, device=self.dev)
        self.order[n : n + T] = torch.arange(n, n + T, dtype=torch.int32, device=self.dev)
        self.args.n_traj = n + T
        if self._n != n:
            self._graph = None
        self._n = n

    def autotune(self, y0: torch.Tensor, path: str | None = None, force: bool = False, **kw):
        """Pick the integrator's launch shape (block size, grid, dense mode, schedule,
        refill threshold) by timing candidate passes over device ICs ``y0``; the
        result is cached per workload signature (in memory, and in ``path`` when
        given) and left configured on this pipeline.  Returns the ``TuneResult``
        (its ``tune_s`` is the tuning time, kept out of any timed pass)."""
        from pybasin_b200.autotune import tune_pipeline

        return tune_pipeline(self, y0, path=path, force=force, **kw)

    # -- one pass ----------------------------------------------------------------
    def _launch(self) -> None:
        lib = L.load()
        s = ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        launch_solve(lib, self.args, self.program, s.value or 0)
        n = self._n
        assert n is not None
        feats = self.out.features
        rc = lib.pb_label_nearest(
            feats.data_ptr(),
            n,
            feats.shape[1],
            feats[n:].data_ptr(),
            self.n_tpl,
            self.tpl_class.data_ptr(),
            self.n_classes,
            self.out.status.data_ptr(),
            self.pidx.data_ptr() if self.n_groups > 1 else None,
            self.n_groups,
            self.labels.data_ptr(),
            self.counts.data_ptr(),
            s,
        )
        L.check(rc, "pb_label_nearest")

    def kernel_launches_per_pass(self) -> int:
        """Launches of this library's own kernels per pass (CUB radix-sort passes not
        counted): the Z-order (bounding box, keys, index fill), then integrate
        (inline), or integrate + sample + redo of record overflows (deferred, with
        the FP32 split of the save grid in mixed precision; the probed schedule
        integrates in a probe and a main launch), then labelling."""
        deferred = self.solver.dense_mode == "deferred"
        n = 3 if self.solver.order == "morton" else 0
        if not deferred:
            return n + 2
        split = 1 if self.solver.precision != "fp64" else 0
        return n + split + (5 if self.solver.schedule == "probed" else 4)

    def load_rows(self, y0: torch.Tensor, group: torch.Tensor | None = None) -> int:
        """Copy device ICs (and their parameter points) into the pipeline, growing it if needed."""
        n = y0.shape[0]
        if group is None and self.n_groups > 1:
            raise ValueError("a parameter study needs the parameter point (group) of every IC")
        if group is not None and group.shape[0] != n:
            raise ValueError("group must hold one entry per IC")
        if getattr(self, "capacity", -1) < n:
            self._allocate(n)
        self.y0_buf[:n].copy_(y0, non_blocking=True)
        self._prepare(n, group)
        return n

    def run_device(
        self, y0: torch.Tensor, use_graph: bool = False, group: torch.Tensor | None = None
    ) -> tuple[torch.Tensor, torch.Tensor]:
        """Label device-resident ``y0`` (N, S) on the current stream; asynchronous.

        Returns labels (N,) int32 and counts (P, n_classes + 1) int64 (last column:
        unbounded).  With a parameter study, ``group`` (N,) gives each IC's point."""
        n = self.load_rows(y0, group)
        if use_graph:
            if self._graph is None:
                self._capture()
            assert self._graph is not None
            self._graph.replay()
        else:
            self._launch()
        return self.labels[:n], self.counts

    def _capture(self) -> None:
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self._launch()  # warm-up outside capture (lazy module loading)
        s.synchronize()
        with torch.cuda.graph(g, stream=s):
            self._launch()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        self._graph = g

    def run(self, y0_host: torch.Tensor, use_graph: bool = False, names: bool = True
            ) -> tuple[np.ndarray, dict[str, float]]:
        """Host ICs -> (labels, basin stability per class); labels as class names, or
        with ``names=False`` as int32 indices into ``classes + ["unbounded"]``."""
        with torch.cuda.device(self.dev):
            y0 = y0_host.to(self.dev, dtype=torch.float32, non_blocking=True)
            labels, counts = self.run_device(y0, use_graph=use_graph)
            lab, cnt_all = to_host_pinned(self, labels, counts)
            cnt = cnt_all.reshape(counts.shape)[0]
        classes = np.array(self.classes + ["unbounded"], dtype=object)
        n = max(int(cnt.sum()), 1)
        bs = {classes[i]: float(cnt[i]) / n for i in range(len(classes)) if cnt[i] > 0}
        return (classes[lab] if names else lab.copy()), bs
