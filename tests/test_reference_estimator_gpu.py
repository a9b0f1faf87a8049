"""The reference's own BasinStabilityEstimator driving the drop-in solver.

src/pybasin/basin_stability_estimator.py:488-517 integrates the main ICs and the
templates concurrently in a two-thread pool; src/pybasin/template_integrator.py:
80-103 clones the solver to the CPU for the templates; src/pybasin/solution.py:
56-68 asserts the shapes; the feature extractor reads the features through the
solution.  Here all of that runs unmodified, on pendulum case 1 (seed 42, N =
4000), with B200Dopri5Solver + FusedFeatureExtractor in place of the reference's
solver and extractor, and the basin stability must equal the reference's fixture
(tests/integration/pendulum/main_pendulum_case1.json: FP 602, LC 3398).

The reference tree is read from PYBASIN_REFERENCE (its root) with empty
stand-ins for the two imports that are not installed (torchdiffeq,
matplotlib).  The test needs both that tree and a GPU, so it is skipped where
either is missing.
"""

from __future__ import annotations

import os
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _reference_tree() -> Path | None:
    root = os.environ.get("PYBASIN_REFERENCE")
    if not root:
        return None
    p = Path(root)
    return p if (p / "src" / "pybasin" / "basin_stability_estimator.py").exists() else None


def _stand_ins() -> None:
    tmp = Path(tempfile.mkdtemp(prefix="pb_stand_ins_"))
    (tmp / "torchdiffeq").mkdir()
    (tmp / "torchdiffeq" / "__init__.py").write_text("def odeint(*a, **k):\n    raise RuntimeError('absent')\n")
    mpl = tmp / "matplotlib"
    mpl.mkdir()
    (mpl / "__init__.py").write_text("def use(*a, **k):\n    pass\n")
    for mod in ("pyplot", "colors"):
        (mpl / f"{mod}.py").write_text("def __getattr__(name):\n    raise AttributeError(name)\n")
    (mpl / "figure.py").write_text("class Figure: pass\n")
    (mpl / "axes.py").write_text("class Axes: pass\n")
    sys.path.insert(0, str(tmp))


def test_reference_estimator_runs_the_drop_in_on_pendulum_case1():
    ref = _reference_tree()
    if ref is None:
        pytest.skip("the reference tree is not present (set PYBASIN_REFERENCE to its root)")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    _stand_ins()
    sys.path.insert(0, str(ref / "src"))
    from sklearn.neighbors import KNeighborsClassifier

    from pybasin.basin_stability_estimator import BasinStabilityEstimator
    from pybasin.sampler import UniformRandomSampler
    from pybasin.template_integrator import TemplateIntegrator
    from pybasin_b200 import B200Dopri5Solver, FusedFeatureExtractor, PendulumODE

    params = {"alpha": 0.1, "T": 0.5, "K": 1.0}
    torch.manual_seed(42)
    sampler = UniformRandomSampler(min_limits=[-np.pi + np.arcsin(0.5), -10.0],
                                   max_limits=[np.pi + np.arcsin(0.5), 10.0], device="cpu")
    fx = FusedFeatureExtractor(time_steady=950.0, features=None, features_per_state={1: {"log_delta": None}},
                               normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=1000, device="cuda:0", rtol=1e-8, atol=1e-6,
                              precision="fp64", feature_extractor=fx)
    bse = BasinStabilityEstimator(
        n=4000, ode_system=PendulumODE(params), sampler=sampler, solver=solver, feature_extractor=fx,
        predictor=KNeighborsClassifier(n_neighbors=1),
        template_integrator=TemplateIntegrator(template_y0=[[0.4, 0.0], [2.7, 0.0]], labels=["FP", "LC"],
                                               ode_params=params),
        feature_selector=None,
    )
    res = bse.run()
    bs = res["basin_stability"]
    want = np.load(GOLDEN / "labels_pendulum_case1.npz")["counts"]
    assert round(bs["FP"] * 4000) == int(want[0]) and round(bs["LC"] * 4000) == int(want[1])
