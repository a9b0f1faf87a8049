"""The launch-shape autotuner: candidate shapes, the cache, and (GPU) a tuning run
whose chosen shape gives the same outputs as the untuned pipeline, bit for bit.
Every launch shape integrates every trajectory with the same step sequence, so the
features, step counts and labels do not depend on the shape."""

from __future__ import annotations

import json

import pytest
import torch

from pybasin_b200 import autotune as A


def test_candidates_cover_every_knob_and_are_valid():
    c = A.candidate_shapes(100_000, 148)
    assert {s.block_size for s in c} == {64, 128, 256}
    assert {s.schedule for s in c} == {"queue", "probed"}
    assert {s.refill_lanes for s in c} == {32, 16, 8}
    assert all(s.dense_mode == "deferred" for s in c)
    for s in c:
        assert s.block_size % 32 == 0 and 0 < s.block_size <= 256
        assert s.grid_blocks == 0 or s.grid_blocks >= 148
        assert 1 <= s.refill_lanes <= 32
    assert len(set(c)) == len(c)
    # inline dense output only with the queue schedule (the probed one needs step records)
    c2 = A.candidate_shapes(10_000, 148, dense_modes=("deferred", "inline"))
    assert not any(s.schedule == "probed" and s.dense_mode == "inline" for s in c2)
    # a small batch: no reduced grid below one wave
    c3 = A.candidate_shapes(1000, 148)
    assert all(s.grid_blocks == 0 for s in c3)


def test_cache_entries_round_trip(tmp_path):
    best = A.LaunchShape(64, 0, "deferred", "probed", 16)
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"k": {"best": A.asdict(best), "best_ms": 1.5}}))
    loaded = A._load(path)
    assert A.LaunchShape(**loaded["k"]["best"]) == best
    assert A._load(tmp_path / "missing.json") == {}


@pytest.mark.gpu
def test_tuning_picks_a_shape_with_identical_outputs(tmp_path):
    from tests.helpers import DUFFING, seeded_ics
    from pybasin_b200 import B200Dopri5Solver, DuffingODE, FusedFeatureExtractor
    from pybasin_b200.pipeline import BasinStabilityPipeline

    dev = torch.device("cuda:0")

    def pipeline():
        fx = FusedFeatureExtractor(time_steady=900.0, features=None,
                                   features_per_state={0: {"maximum": None, "standard_deviation": None}},
                                   normalize=False)
        solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=5000, t_eval=(900, 1000), device="cuda:0",
                                  precision="mixed", feature_extractor=fx)
        return BasinStabilityPipeline(DuffingODE(dict(zip(("delta", "k3", "A"), DUFFING.params))), solver,
                                      [list(t) for t in DUFFING.templates], ["y1", "y2", "y3", "y4", "y5"], device=dev)

    y0 = seeded_ics(DUFFING, 6000, seed=9).to(dev)
    ref = pipeline()
    ref.run_device(y0)
    torch.cuda.synchronize()
    ref_feat, ref_steps, ref_lab = ref.out.features[:6000].clone(), ref.out.steps[:6000].clone(), ref.labels.clone()

    pipe = pipeline()
    cands = [A.LaunchShape(64, 0, "deferred", "probed", 32), A.LaunchShape(128, 0, "deferred", "queue", 8),
             A.LaunchShape(64, 0, "deferred", "probed", 16), A.LaunchShape(256, 60, "deferred", "queue", 32)]
    res = pipe.autotune(y0, path=str(tmp_path / "tune.json"), candidates=cands, repeats=1, force=True)
    assert res.best in cands and res.tune_s > 0 and len(res.table) == len(cands)
    for shape in cands:  # every candidate: the same outputs, bit for bit
        A._apply(pipe, shape)
        pipe.run_device(y0)
        torch.cuda.synchronize()
        assert torch.equal(pipe.out.features[:6000], ref_feat), shape
        assert torch.equal(pipe.out.steps[:6000], ref_steps), shape
        assert torch.equal(pipe.labels[:6000], ref_lab[:6000]), shape
    # the cached result is reused without timing
    again = pipe.autotune(y0, path=str(tmp_path / "tune.json"))
    assert again.best == res.best and again.tune_s == 0.0
