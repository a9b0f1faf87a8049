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
