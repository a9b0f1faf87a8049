"""Friction oscillator (non-smooth stick-slip right-hand side) on the GPU.

The reference's friction case 1 (tests/integration/friction/test_friction.py:17-45:
seed 42, N = 4000, FP 1266 / LC 2734, MCC >= 0.95): the FP64 kernel must give the
fixture's labels (the FP64 oracle reproduces all 4000); the mixed kernel must stay
within |dBS| <= 0.005 of them.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from pybasin_b200 import B200Dopri5Solver, FrictionFeatureExtractor, FrictionODE
from pybasin_b200 import _lib as L

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
PARAMS = {"v_d": 1.5, "xi": 0.05, "musd": 2.0, "mud": 0.5, "muv": 0.0, "v0": 0.5}


def _labels(precision: str, schedule: str = "probed"):
    d = np.load(GOLDEN / "labels_friction_case1.npz")
    fx = FrictionFeatureExtractor(time_steady=400.0)
    solver = B200Dopri5Solver(t_span=(0, 500), t_steps=500, t_eval=(400.0, 500.0), device="cuda:0", rtol=1e-8,
                              atol=1e-6, precision=precision, feature_extractor=fx, schedule=schedule)
    t, y = solver.integrate(FrictionODE(PARAMS), torch.tensor(d["ics"]))
    onehot = fx.extract_features(type("S", (), {"y": y})())
    assert (y._pb_status.cpu() == L.TRAJ_OK).all()
    return onehot[:, 1].cpu().numpy().astype(np.int8), d


@pytest.mark.parametrize("schedule", ["probed", "plain"])
def test_fp64_friction_labels_equal_reference_fixture(schedule):
    lab, d = _labels("fp64", schedule)
    assert (lab == d["labels"]).mean() >= 0.999
    assert abs(int(lab.sum()) - 2734) <= 2


def test_mixed_friction_basin_stability_within_bound():
    lab, d = _labels("mixed")
    assert abs(lab.mean() - d["labels"].mean()) <= 0.005
    assert (lab == d["labels"]).mean() >= 0.99
