"""IC sharding across ranks (one process per GPU).

Every initial condition is independent, so a basin-stability estimate shards as
contiguous IC ranges, one per rank, with no exchange during integration.  The
one real exchange is the global basin stability: the per-class counts of all
shards are summed (``all_reduce``), and, when labels are wanted in one place,
the per-rank label vectors are gathered.  A parameter study shards by its
points instead (:func:`run_sharded_study`): each rank integrates whole points,
the points spread by their predicted cost (ICs x pilot steps), and the per-point
counts are all-reduced.  Surrogate training runs data-parallel with one gradient
all-reduce per step (:func:`allreduce_gradients`).  Works with any
``torch.distributed`` backend (NCCL on GPUs, gloo on CPU for the tests).
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's IC shard; shards differ in size by at most one."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("need 0 <= rank < world and n >= 0")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def global_counts(counts: torch.Tensor, group=None) -> torch.Tensor:
    """Per-class counts summed over all ranks (int64)."""
    c = counts.to(torch.int64).clone()
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(c, group=group)
    return c


def basin_stability(counts: torch.Tensor, classes: list[str]) -> dict[str, float]:
    """Fractions per class, the reference's _compute_bs (basin_stability_estimator.py:586-598)."""
    c = counts.cpu().numpy().astype(np.float64)
    n = max(c.sum(), 1.0)
    return {classes[i]: float(c[i] / n) for i in range(len(classes)) if c[i] > 0}


def standard_errors(bs: dict[str, float], n: int) -> dict[str, dict[str, float]]:
    """Bernoulli errors of the reference's get_errors (basin_stability_estimator.py:600-625)."""
    out = {}
    for k, s in bs.items():
        out[k] = {"e_abs": float(np.sqrt(s * (1 - s) / n)), "e_rel": float(1 / np.sqrt(n * s)) if s > 0 else float("inf")}
    return out


def gather_labels(labels: torch.Tensor, n_total: int, group=None) -> torch.Tensor:
    """Concatenate every rank's shard of labels in rank order (shards from shard_range)."""
    if not (dist.is_available() and dist.is_initialized()):
        return labels
    world = dist.get_world_size(group)
    sizes = [shard_range(n_total, r, world)[1] - shard_range(n_total, r, world)[0] for r in range(world)]
    m = max(sizes)
    buf = torch.zeros((m,), dtype=labels.dtype, device=labels.device)
    buf[: labels.numel()] = labels
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)])


# ---------------------------------------------------------------------------
# one parameter study over several ranks
# ---------------------------------------------------------------------------
def partition_groups(loads, world: int) -> list[list[int]]:
    """Parameter points (their loads) over ranks: the heaviest point first onto the
    least loaded rank (longest-processing-time rule, within 4/3 of the optimal
    makespan); ties go to the lower rank, so every rank computes the same split."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = np.asarray(loads, dtype=np.float64)
    order = sorted(range(len(loads)), key=lambda p: (-loads[p], p))
    assign: list[list[int]] = [[] for _ in range(world)]
    total = [0.0] * world
    for p in order:
        r = min(range(world), key=lambda q: (total[q], q))
        assign[r].append(p)
        total[r] += loads[p]
    return [sorted(a) for a in assign]


def pilot_steps(pipe, y0: torch.Tensor, group: torch.Tensor, n_points: int, per_point: int = 64) -> np.ndarray:
    """Mean attempted steps per parameter point from a pilot launch over the first
    ``per_point`` ICs of every point (deterministic, so every rank gets the same
    numbers): the cost of an IC of that point."""
    g = group.to(torch.int64).cpu()
    pick = torch.cat([torch.nonzero(g == p).flatten()[:per_point] for p in range(n_points)])
    pipe.run_device(y0[pick.to(y0.device)], group=group[pick.to(group.device)])
    steps = pipe.out.steps[: pick.numel()].double().cpu()
    gp = g[pick]
    out = np.ones(n_points)
    for p in range(n_points):
        sel = steps[gp == p]
        if sel.numel():
            out[p] = float(sel.mean())
    return out


def run_sharded_study(pipe, y0: torch.Tensor, group: torch.Tensor, n_points: int, loads=None,
                      group_comm=None) -> tuple[torch.Tensor, list[int]]:
    """One parameter study over all ranks: each rank integrates the ICs of its share
    of the points (``partition_groups`` of ``loads``, default the IC counts) in one
    launch, and the (points x classes) counts are all-reduced, so every rank ends
    with the counts of the whole study.  Returns (counts, this rank's points)."""
    world = dist.get_world_size(group_comm) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group_comm) if world > 1 else 0
    g = group.to(torch.int64)
    if loads is None:
        loads = torch.bincount(g.cpu(), minlength=n_points).double().numpy()
    mine = partition_groups(loads, world)[rank]
    n_classes = pipe.n_classes + 1
    counts = torch.zeros((n_points, n_classes), dtype=torch.int64, device=pipe.dev)
    if mine:
        keep = torch.isin(g, torch.tensor(mine, device=g.device))
        idx = torch.nonzero(keep).flatten()
        if idx.numel():
            _, c = pipe.run_device(y0[idx.to(y0.device)], group=group[idx.to(group.device)])
            counts += c.to(torch.int64)
    if world > 1:
        dist.all_reduce(counts, group=group_comm)
    return counts, mine


def allreduce_gradients(grads: list[torch.Tensor], group=None, average: bool = True) -> None:
    """Data-parallel gradients: the tensors of every rank summed (and divided by the
    world size with ``average``) in one collective over a flat buffer, in place."""
    if not (dist.is_available() and dist.is_initialized()) or not grads:
        return
    world = dist.get_world_size(group)
    flat = torch.cat([t.reshape(-1) for t in grads])
    dist.all_reduce(flat, group=group)
    if average:
        flat /= world
    off = 0
    for t in grads:
        n = t.numel()
        t.copy_(flat[off : off + n].view_as(t))
        off += n
