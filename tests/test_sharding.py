"""IC sharding and the count / label exchange across ranks, on CPU with gloo (world size 2)."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pybasin_b200.sharding import basin_stability, gather_labels, global_counts, shard_range, standard_errors


@pytest.mark.parametrize("n,world", [(0, 1), (10, 3), (100_000, 8), (7, 8)])
def test_shards_partition_the_range(n, world):
    spans = [shard_range(n, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def test_bs_and_errors_match_reference_formulas():
    bs = basin_stability(torch.tensor([602, 3398]), ["FP", "LC"])
    assert bs == {"FP": 0.1505, "LC": 0.8495}
    err = standard_errors(bs, 4000)
    # tests/integration/pendulum/main_pendulum_case1.json: standardError 0.005653533187308623
    assert abs(err["FP"]["e_abs"] - 0.005653533187308623) < 1e-15


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, n: int, q) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a, b = shard_range(n, rank, world)
        rng = np.random.default_rng(0)
        labels_all = torch.tensor(rng.integers(0, 3, n), dtype=torch.int32)
        mine = labels_all[a:b]
        counts = torch.bincount(mine.long(), minlength=3)
        tot = global_counts(counts)
        gathered = gather_labels(mine, n)
        q.put((rank, tot.tolist(), bool(torch.equal(gathered, labels_all)),
               torch.bincount(labels_all.long(), minlength=3).tolist()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_counts_and_gather_labels():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, 1001, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, tot, same, want in res:
        assert tot == want
        assert same


# ---------------------------------------------------------------------------
# one parameter study over several ranks; data-parallel gradients
# ---------------------------------------------------------------------------
class _StubPipeline:
    """Stands in for BasinStabilityPipeline on the CPU (the split and the exchange
    are under test, not the kernels): class = (x > 0) + (y > 0.5) per IC, step
    count growing with the point index so the points have different costs."""

    n_classes = 3
    dev = torch.device("cpu")

    def run_device(self, y0, group):
        lab = ((y0[:, 0] > 0).int() + (y0[:, 1] > 0.5).int()).to(torch.int32)
        P = 12
        counts = torch.zeros((P, self.n_classes + 1), dtype=torch.int64)
        counts.index_put_((group.long(), lab.long()), torch.ones_like(lab, dtype=torch.int64), accumulate=True)
        self.out = type("Out", (), {"steps": (100 + 40 * group.long() + (y0[:, 0].abs() * 10).long())})()
        return lab, counts


def _study(seed=1):
    g = torch.Generator().manual_seed(seed)
    counts = [50, 400, 120, 60, 900, 30, 300, 75, 10, 500, 220, 90]
    y0 = torch.rand(sum(counts), 2, generator=g) * 2 - 1
    group = torch.cat([torch.full((c,), p, dtype=torch.int32) for p, c in enumerate(counts)])
    return y0, group, counts


def test_partition_balances_loads():
    from pybasin_b200.sharding import partition_groups

    loads = [5, 1, 1, 1, 1, 1, 4, 3]
    parts = partition_groups(loads, 2)
    assert sorted(sum(parts, [])) == list(range(8))
    tot = [sum(loads[p] for p in part) for part in parts]
    assert max(tot) <= (4 / 3) * (sum(loads) / 2) + max(loads) / 3
    assert partition_groups(loads, 2) == parts  # deterministic
    assert partition_groups([1, 2, 3], 5)[3:] == [[], []]


def _study_worker(rank: int, world: int, port: int, q) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pybasin_b200.sharding import allreduce_gradients, pilot_steps, run_sharded_study

        pipe = _StubPipeline()
        y0, group, counts = _study()
        steps = pilot_steps(pipe, y0, group, 12)
        loads = np.array(counts) * steps
        tot, mine = run_sharded_study(pipe, y0, group, 12, loads=loads)
        # data-parallel gradients: every rank ends with the mean of all ranks' tensors
        grads = [torch.full((3, 4), float(rank + 1)), torch.arange(5, dtype=torch.float32) * (rank + 1)]
        allreduce_gradients(grads)
        q.put((rank, tot.tolist(), mine, loads.tolist(), grads[0].tolist(), grads[1].tolist()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_one_study_and_average_gradients():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_study_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    y0, group, _ = _study()
    _, want = _StubPipeline().run_device(y0, group)
    (r0, tot0, mine0, loads, g00, g01), (r1, tot1, mine1, _, g10, g11) = res
    assert tot0 == want.tolist() and tot1 == want.tolist()  # every rank has the whole study
    assert sorted(mine0 + mine1) == list(range(12)) and not set(mine0) & set(mine1)
    l0, l1 = sum(loads[p] for p in mine0), sum(loads[p] for p in mine1)
    assert max(l0, l1) <= (4 / 3) * (sum(loads) / 2) + max(loads) / 3
    assert g00 == g10 == [[1.5] * 4] * 3
    assert g01 == g11 == [0.0, 1.5, 3.0, 4.5, 6.0]
