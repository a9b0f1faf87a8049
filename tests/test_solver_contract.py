"""SolverProtocol contract of B200Dopri5Solver, mirroring the reference's
tests/unit/solvers/test_solver.py (:30-249) plus the fused side channel.

Construction-time behaviour needs no GPU; integration tests are marked gpu.
"""

from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
import torch

from pybasin_b200 import B200Dopri5Solver, FusedFeatureExtractor, LinearODE, PendulumODE, register_system
from pybasin_b200.odes import resolve_system


class ExponentialDecayODE(LinearODE):
    """The reference test's ODE: dy/dt = decay * y (test_solver.py:16-21)."""

    def get_str(self) -> str:
        return f"dy/dt = {self.params['decay']} * y"


@pytest.fixture
def simple_ode() -> ExponentialDecayODE:
    return ExponentialDecayODE({"decay": -1.0})


# ---- construction (CPU) -----------------------------------------------------
@pytest.mark.parametrize("t_eval", [(0.5, 1.5), (-1.0, 0.5)])
def test_t_eval_out_of_span_raises(t_eval):
    with pytest.raises(ValueError, match="t_eval"):
        B200Dopri5Solver(t_span=(0, 1), t_steps=10, t_eval=t_eval, device="cpu", cache_dir=None)


def test_t_eval_propagates_to_clone():
    solver = B200Dopri5Solver(t_span=(0, 2), t_steps=10, t_eval=(1, 2), device="cpu", cache_dir=None)
    cloned = solver.clone(device="cpu", cache_dir=None)
    assert cloned.t_eval == (1, 2)
    assert cloned.clone(t_steps_factor=3).t_steps == 30


def test_device_normalisation():
    assert B200Dopri5Solver(device="cuda").device == torch.device("cuda:0")
    assert B200Dopri5Solver(device="cuda:1").device == torch.device("cuda:1")
    assert B200Dopri5Solver(device="cpu").device == torch.device("cpu")


def test_protocol_surface_matches_reference_signature():
    import inspect

    sig = inspect.signature(B200Dopri5Solver.__init__)
    names = list(sig.parameters)[1:9]
    assert names == ["t_span", "t_steps", "device", "method", "rtol", "atol", "cache_dir", "t_eval"]
    assert sig.parameters["rtol"].default == 1e-8 and sig.parameters["atol"].default == 1e-6
    csig = inspect.signature(B200Dopri5Solver.clone)
    assert {"device", "t_steps_factor", "cache_dir"} <= set(csig.parameters)


def test_bad_options_raise():
    with pytest.raises(ValueError):
        B200Dopri5Solver(method="rk4")
    with pytest.raises(ValueError):
        B200Dopri5Solver(precision="fp16")
    with pytest.raises(ValueError):
        B200Dopri5Solver(output="fused")  # needs an extractor


def test_system_resolution_by_class_name_and_registry():
    class PendulumJaxODE:  # reference class name, no torch needed
        params = {"alpha": 0.1, "T": 0.5, "K": 1.0}

    spec = resolve_system(PendulumJaxODE(), 2)
    assert spec.params.tolist() == [0.1, 0.5, 1.0]

    class MyDecay:
        params = {"k": -0.5}

    with pytest.raises(ValueError, match="no B200 right-hand side"):
        resolve_system(MyDecay(), 1)
    register_system(MyDecay, "linear")
    assert resolve_system(MyDecay(), 1).params.tolist() == [-0.5]
    with pytest.raises(ValueError, match="dimension"):
        resolve_system(PendulumODE({"alpha": 0.1, "T": 0.5, "K": 1.0}), 3)


def test_feature_columns_and_names_follow_reference_order():
    fx = FusedFeatureExtractor(
        time_steady=900.0, features=None, features_per_state={0: {"maximum": None, "standard_deviation": None}}
    )
    cols = fx.columns(2)
    assert [c.name for c in cols] == ["state_0__maximum", "state_0__standard_deviation"]
    fx2 = FusedFeatureExtractor(features={"mean": None, "number_crossing_m": [{"m": 0}, {"m": 1}]})
    assert [c.name for c in fx2.columns(2)] == [
        "state_0__mean",
        "state_0__number_crossing_m__m_0",
        "state_0__number_crossing_m__m_1",
        "state_1__mean",
        "state_1__number_crossing_m__m_0",
        "state_1__number_crossing_m__m_1",
    ]
    with pytest.raises(ValueError, match="fused statistics"):
        FusedFeatureExtractor(features={"sample_entropy": None}).columns(1)
    # attribute-selected kernels keep the reference's parameter names
    fft = FusedFeatureExtractor(features={"fft_coefficient": [{"coeff": 2, "attr": "imag"}],
                                          "linear_trend": [{"attr": "stderr"}]}).columns(1)
    assert [c.name for c in fft] == ["state_0__fft_coefficient__attr_imag__coeff_2",
                                     "state_0__linear_trend__attr_stderr"]
    with pytest.raises(ValueError, match="attr"):
        FusedFeatureExtractor(features={"linear_trend": [{"attr": "slop"}]}).columns(1)


def test_y0_shape_validation_before_any_gpu_work(simple_ode):
    solver = B200Dopri5Solver(t_span=(0, 1), t_steps=10, device="cpu", cache_dir=None)
    with pytest.raises(ValueError, match="y0 must be 2D with shape"):
        solver.integrate(simple_ode, torch.tensor([1.0]))
    with pytest.raises(ValueError, match="y0 must be 2D with shape"):
        solver.integrate(simple_ode, torch.tensor([[[1.0]]]))


# ---- integration (GPU) ------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_integration_single(simple_ode, precision):
    solver = B200Dopri5Solver(t_span=(0, 1), t_steps=10, device="cpu", cache_dir=None, precision=precision)
    t, y = solver.integrate(simple_ode, torch.tensor([[1.0]]))
    assert t.shape == (10,)
    assert y.shape == (10, 1, 1)
    assert y[0].item() == pytest.approx(1.0, abs=1e-5)
    assert y[-1].item() < y[0].item()
    assert y[-1].item() == pytest.approx(np.exp(-1.0), abs=1e-5)


@pytest.mark.gpu
def test_batched_ratio_preserved(simple_ode):
    solver = B200Dopri5Solver(t_span=(0, 1), t_steps=10, device="cuda", cache_dir=None)
    t, y = solver.integrate(simple_ode, torch.tensor([[1.0], [2.0]]))
    assert t.shape == (10,) and y.shape == (10, 2, 1)
    assert torch.allclose(y[:, 1, :] / y[:, 0, :], torch.tensor([[2.0]], device=y.device), atol=1e-5)


@pytest.mark.gpu
def test_t_eval_saves_only_subrange(simple_ode):
    solver = B200Dopri5Solver(t_span=(0, 2), t_steps=10, t_eval=(1, 2), device="cpu", cache_dir=None)
    t, y = solver.integrate(simple_ode, torch.tensor([[1.0]]))
    assert t.shape == (10,) and y.shape == (10, 1, 1)
    assert t[0].item() == pytest.approx(1.0, abs=1e-5)
    assert t[-1].item() == pytest.approx(2.0, abs=1e-5)
    assert y[0].item() == pytest.approx(0.368, abs=0.01)


@pytest.mark.gpu
def test_params_batched(simple_ode):
    solver = B200Dopri5Solver(t_span=(0, 1), t_steps=11, device="cpu", cache_dir=None)
    _, y = solver.integrate(simple_ode, torch.tensor([[1.0]]), params=torch.tensor([[-1.0], [-2.0]]))
    assert y.shape == (11, 2, 1)
    assert y[0, 0, 0].item() == pytest.approx(1.0, abs=1e-5)
    assert y[0, 1, 0].item() == pytest.approx(1.0, abs=1e-5)
    assert y[-1, 1, 0].item() < y[-1, 0, 0].item()
    assert y[-1, 0, 0].item() == pytest.approx(0.368, abs=0.01)
    assert y[-1, 1, 0].item() == pytest.approx(0.135, abs=0.01)


@pytest.mark.gpu
def test_params_ic_major_order():
    """Row ic*P + p carries (y0[ic], params[p]) (src/pybasin/solvers/base.py:155-159)."""
    ode = ExponentialDecayODE({"decay": -1.0})
    solver = B200Dopri5Solver(t_span=(0, 1), t_steps=2, device="cpu", cache_dir=None)
    y0 = torch.tensor([[1.0], [3.0]])
    params = torch.tensor([[-1.0], [-2.0], [-3.0]])
    _, y = solver.integrate(ode, y0, params=params)
    want = torch.tensor([y0[ic, 0] * np.exp(params[p, 0]) for ic in range(2) for p in range(3)])
    assert torch.allclose(y[-1, :, 0].double(), want.double(), atol=1e-5)


@pytest.mark.gpu
def test_fused_mode_side_channel_and_templates_on_cpu():
    """Fused output: compact y, features attached; a CPU clone (TemplateIntegrator,
    template_integrator.py:80-86) still computes on the GPU and returns CPU tensors."""
    fx = FusedFeatureExtractor(time_steady=950.0, features=None, features_per_state={1: {"log_delta": None}},
                               normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=1000, device="cuda", feature_extractor=fx, cache_dir=None)
    ode = PendulumODE({"alpha": 0.1, "T": 0.5, "K": 1.0})
    y0 = torch.tensor([[0.4, 0.0], [2.7, 0.0]], device="cuda")
    res = solver.integrate(ode, y0)
    t, y = res
    assert t.shape == (1,) and y.shape == (1, 2, 2)
    from types import SimpleNamespace

    feats = fx.extract_features(SimpleNamespace(y=y, time=t))
    assert feats.shape == (2, 1) and fx.feature_names == ["state_1__log_delta"]
    assert feats[0, 0] < -10 and feats[1, 0] > -5  # fixed point vs rotating limit cycle
    cpu = solver.clone(device="cpu")
    t2, y2 = cpu.integrate(ode, y0.cpu())
    assert y2.device.type == "cpu"
    f2 = fx.extract_features(SimpleNamespace(y=y2, time=t2))
    assert torch.allclose(f2, feats.cpu())


@pytest.mark.gpu
def test_concurrent_integrations_from_two_threads():
    """The estimator integrates main and template sets concurrently (bse.py:499-512)."""
    ode = PendulumODE({"alpha": 0.1, "T": 0.5, "K": 1.0})
    fx = FusedFeatureExtractor(time_steady=950.0, features=None, features_per_state={1: {"log_delta": None}},
                               normalize=False)
    solver = B200Dopri5Solver(feature_extractor=fx, device="cuda", cache_dir=None)
    torch.manual_seed(0)
    y0 = torch.rand(2000, 2) * 6 - 3
    ref = solver.integrate(ode, y0.cuda()).features
    with ThreadPoolExecutor(max_workers=2) as ex:
        a = ex.submit(solver.integrate, ode, y0.cuda())
        b = ex.submit(solver.clone(device="cpu").integrate, ode, y0)
        fa, fb = a.result().features, b.result().features
    assert torch.equal(fa, ref)
    assert torch.equal(fb, ref.cpu())


@pytest.mark.gpu
def test_unbounded_rows_are_inf_in_fused_mode():
    fx = FusedFeatureExtractor(features={"mean": None}, normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 10), t_steps=11, feature_extractor=fx, unbounded_threshold=1e6,
                              device="cuda", cache_dir=None)
    ode = ExponentialDecayODE({"decay": 5.0})
    res = solver.integrate(ode, torch.tensor([[1.0], [0.0]], device="cuda"))
    _, y = res
    assert torch.isinf(y[0, 0, 0]) and not torch.isinf(y[0, 1, 0])
    assert res.status.tolist() == [3, 0]


@pytest.mark.gpu
def test_result_cache_roundtrip():
    """Second call with the same inputs is served from the safetensors cache
    (src/pybasin/cache_manager.py:27-128); other inputs miss."""
    import shutil
    from pathlib import Path

    from pybasin_b200 import B200Dopri5Solver, DuffingODE, FusedFeatureExtractor

    cache = Path(__file__).resolve().parent / "_cache_roundtrip"
    shutil.rmtree(cache, ignore_errors=True)
    try:
        fx = FusedFeatureExtractor(time_steady=90.0, features=None,
                                   features_per_state={0: {"maximum": None}}, normalize=False)
        solver = B200Dopri5Solver(t_span=(0, 100), t_steps=200, device="cuda:0", precision="mixed",
                                  feature_extractor=fx, cache_dir=str(cache))
        ode = DuffingODE({"delta": 0.08, "k3": 1.0, "A": 0.2})
        y0 = torch.rand(64, 2, generator=torch.Generator().manual_seed(1))
        t1, y1 = solver.integrate(ode, y0)
        files = list(cache.glob("*.safetensors"))
        assert len(files) == 1
        t2, y2 = solver.integrate(ode, y0)
        assert torch.equal(y1.cpu(), y2.cpu()) and torch.equal(y1._pb_features.cpu(), y2._pb_features.cpu())
        solver.integrate(ode, y0 + 0.01)
        assert len(list(cache.glob("*.safetensors"))) == 2
    finally:
        shutil.rmtree(cache, ignore_errors=True)
