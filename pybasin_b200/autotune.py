"""Launch-shape autotuner for the integrator pass.

Per workload signature (device, system, state dimension, precision, batch size
rounded to a power of two, window length) it times candidate launch shapes of
one full pass on the caller's own ICs and keeps the fastest:

* ``block_size`` — threads per block of the integrator kernel;
* ``grid_blocks`` — persistent blocks of the queue schedule.  One block per 4
  warps of work gives every warp exactly one 32-trajectory task (no dynamic
  balancing: an SM whose tasks happen to be long finishes last); fewer blocks
  make warps come back to the queue, which balances the SMs at the price of
  fewer warps in flight;
* ``dense_mode`` — deferred (step records + sampling pass) or inline;
* ``schedule`` — the queue in processing order, or probed (a probe over the
  first 5 % of the span orders the trajectories longest first);
* ``refill_lanes`` — the queue depth of a warp: it fetches new queue positions
  for its idle lanes once this many of its 32 lanes are idle (32: only a fully
  idle warp refills; fewer: lanes whose trajectories finished early or stopped
  take new work while the rest of the warp integrates).

Lanes per trajectory are not a knob for the built-in systems: a trajectory of
two or three states is one serial chain of stages (splitting it over lanes
adds shuffles to every stage and leaves lanes idle), and the network systems
take one warp per trajectory with their nodes spread over its lanes, the
register budget bounding the nodes per lane.

Tuning time is reported, never part of a timed pass.  Results are cached in
memory and, with ``path``, in a JSON file.
"""

from __future__ import annotations

import json
import math
import statistics
import time
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Any

import torch


@dataclass(frozen=True)
class LaunchShape:
    block_size: int
    grid_blocks: int  # 0 = one block per block_size trajectories (every warp one task)
    dense_mode: str  # "deferred" | "inline"
    schedule: str = "queue"  # "queue" | "probed"
    refill_lanes: int = 32  # idle lanes of a warp that trigger a refill from the queue


@dataclass
class TuneResult:
    best: LaunchShape
    best_ms: float
    table: list[tuple[LaunchShape, float]] = field(default_factory=list)
    tune_s: float = 0.0
    key: str = ""


def sm_count(dev: torch.device) -> int:
    return torch.cuda.get_device_properties(dev).multi_processor_count


def candidate_shapes(
    n_traj: int,
    sms: int,
    dense_modes: tuple[str, ...] = ("deferred",),
    schedules: tuple[str, ...] = ("queue", "probed"),
    refills: tuple[int, ...] = (32, 16, 8),
    block_sizes: tuple[int, ...] = (64, 128, 256),
) -> list[LaunchShape]:
    """Block sizes x grids from one task per warp down to ~1.5 SM-waves x refill
    thresholds (the refill only matters where warps come back to the queue, so the
    smaller thresholds are paired with the full grid of each block size)."""
    out: list[LaunchShape] = []
    for sched in schedules:
        for mode in dense_modes:
            if sched == "probed" and mode != "deferred":
                continue  # the probed schedule applies to deferred dense output
            for bs in block_sizes:
                need = math.ceil(n_traj / bs)
                grids = {0}
                for frac in (0.75, 0.5, 0.33, 0.25):
                    g = int(need * frac)
                    if g >= sms:
                        grids.add(g)
                for g in sorted(grids, reverse=True):
                    out.append(LaunchShape(bs, g, mode, sched, 32))
                for r in refills:
                    if r != 32:
                        out.append(LaunchShape(bs, 0, mode, sched, r))
    return out


def signature(pipe: Any, n: int) -> str:
    props = torch.cuda.get_device_properties(pipe.dev)
    n_bucket = 1 << max(0, (n - 1).bit_length())
    win = int(pipe.save_ts.shape[0] - pipe.win_begin)
    return f"{props.name}|sys{pipe.spec.system}|S{pipe.dim}|{pipe.solver.precision}|n{n_bucket}|w{win}"


_MEMO: dict[str, dict] = {}


def _load(path: Path | None) -> dict[str, dict]:
    if path is None or not path.exists():
        return {}
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _apply(pipe: Any, shape: LaunchShape) -> None:
    pipe.solver.block_size = shape.block_size
    pipe.solver.grid_blocks = shape.grid_blocks
    if pipe.solver.dense_mode != shape.dense_mode or pipe.solver.schedule != shape.schedule:
        pipe.solver.dense_mode = shape.dense_mode
        pipe.solver.schedule = shape.schedule
        pipe._allocate(pipe.capacity)  # the scratch layout depends on both
    pipe.solver.refill_lanes = shape.refill_lanes
    pipe.args.block_size = shape.block_size
    pipe.args.grid_blocks = shape.grid_blocks
    pipe.args.refill_lanes = shape.refill_lanes
    pipe._graph = None


def _time_pass(pipe: Any, y0: torch.Tensor, repeats: int, warmup: int) -> float:
    for _ in range(warmup):
        pipe.run_device(y0)
    ts = []
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pipe.run_device(y0)
        e1.record()
        torch.cuda.synchronize(pipe.dev)
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def tune_pipeline(
    pipe: Any,
    y0: torch.Tensor,
    candidates: list[LaunchShape] | None = None,
    repeats: int = 3,
    warmup: int = 1,
    path: str | Path | None = None,
    force: bool = False,
) -> TuneResult:
    """Time ``candidates`` on a ``BasinStabilityPipeline`` pass over device ICs ``y0``
    and leave the pipeline configured with the fastest shape."""
    p = Path(path) if path is not None else None
    pipe.load_rows(y0)
    key = signature(pipe, y0.shape[0])
    cache = {**_load(p), **_MEMO}
    if not force and key in cache:
        ent = cache[key]
        best = LaunchShape(**{k: v for k, v in ent["best"].items() if k in LaunchShape.__dataclass_fields__})
        _apply(pipe, best)
        return TuneResult(best, ent["best_ms"], [], 0.0, key)
    if pipe.solver.schedule not in ("queue", "probed"):
        raise ValueError("launch-shape tuning applies to the queue and probed schedules")
    cands = candidates or candidate_shapes(pipe.args.n_traj, sm_count(pipe.dev))
    t0 = time.perf_counter()
    table: list[tuple[LaunchShape, float]] = []
    for shape in cands:
        _apply(pipe, shape)
        table.append((shape, _time_pass(pipe, y0, repeats, warmup)))
    best, best_ms = min(table, key=lambda r: r[1])
    _apply(pipe, best)
    res = TuneResult(best, best_ms, table, time.perf_counter() - t0, key)
    ent = {"best": asdict(best), "best_ms": best_ms}
    _MEMO[key] = ent
    if p is not None:
        disk = _load(p)
        disk[key] = ent
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_text(json.dumps(disk, indent=1, sort_keys=True))
    return res

