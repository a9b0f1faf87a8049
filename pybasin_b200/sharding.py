"""IC sharding across ranks (one process per GPU).

Every initial condition is independent, so a basin-stability estimate shards as
contiguous IC ranges, one per rank, with no exchange during integration.  The
one real exchange is the global basin stability: the per-class counts of all
shards are summed (``all_reduce``), and, when labels are wanted in one place,
the per-rank label vectors are gathered.  Works with any ``torch.distributed``
backend (NCCL on GPUs, gloo on CPU for the tests).
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
