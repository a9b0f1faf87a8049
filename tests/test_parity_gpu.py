"""Parity of the CUDA kernels (through the C ABI) with the FP64 oracle and the golden fixtures.

Tolerances:
* FP64 kernel vs FP64 oracle, short horizon (non-chaotic): rtol 1e-9 on trajectories.
* FP64 kernel vs oracle, full horizon: window features rtol 1e-6 / atol 1e-8 on
  trajectories away from basin boundaries; labels identical on the fixtures.
* Mixed kernel (FP32 stages, rtol 1e-6) vs FP64 oracle: |dBS| <= 0.005 and features
  within 2e-3 relative on the attractors.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pybasin_b200 import _lib as L
from pybasin_b200.engine import FeatureColumn, SolveRequest, label_nearest, solve
from tests.helpers import DUFFING, PENDULUM, Case, impute, knn_labels, oracle_case_features, seeded_ics

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
DEV = torch.device("cuda:0")

SYS_OF = {
    O.SYS_LINEAR: L.SYS_LINEAR,
    O.SYS_PENDULUM: L.SYS_PENDULUM,
    O.SYS_DUFFING: L.SYS_DUFFING,
    O.SYS_LORENZ: L.SYS_LORENZ,
    O.SYS_LORENZ_MASKED: L.SYS_LORENZ_MASKED,
}


def gpu_solve(
    oracle_sys: int,
    y0: np.ndarray,
    params: np.ndarray,
    save: np.ndarray,
    t_span: tuple[float, float],
    rtol: float,
    atol: float,
    *,
    precision: int = L.PREC_FP64,
    schedule: int = L.SCHED_QUEUE,
    win_begin: int = 0,
    features: list[tuple[int, int, float]] | None = None,
    param_index: np.ndarray | None = None,
    layout: int | None = None,
    keep_full: bool = False,
    max_steps: int = 16**5,
    unbounded_thr: float = 0.0,
    y0_dtype=torch.float64,
    block_size: int = 0,
    grid_blocks: int = 0,
    dense_mode: int = L.DENSE_DEFERRED,
    window_record_cap: int = 0,
    refill_lanes: int = 0,
):
    y0_t = torch.as_tensor(np.ascontiguousarray(y0), dtype=y0_dtype, device=DEV)
    p_t = torch.as_tensor(np.ascontiguousarray(np.atleast_2d(params)), dtype=torch.float64, device=DEV)
    if layout is None:
        layout = L.LAYOUT_INDEXED if param_index is not None else L.LAYOUT_SINGLE
    req = SolveRequest(
        system=SYS_OF[oracle_sys],
        dim=y0.shape[1],
        y0=y0_t,
        params=p_t,
        save_ts=torch.as_tensor(save, dtype=torch.float64, device=DEV),
        t_span=t_span,
        rtol=rtol,
        atol=atol,
        layout=layout,
        param_index=None if param_index is None else torch.as_tensor(param_index, dtype=torch.int32, device=DEV),
        win_begin=win_begin,
        columns=[FeatureColumn(f[0], f[1], f[2], "", f[3] if len(f) > 3 else 0.0) for f in (features or [])],
        precision=precision,
        schedule=schedule,
        max_steps=max_steps,
        unbounded_thr=unbounded_thr,
        keep_final=True,
        keep_full=keep_full,
        out_dtype=torch.float64,
        keep_steps=True,
        block_size=block_size,
        grid_blocks=grid_blocks,
        dense_mode=dense_mode,
        window_record_cap=window_record_cap,
        refill_lanes=refill_lanes,
    )
    r = solve(req)
    torch.cuda.synchronize()
    out = {
        "status": r.status.cpu().numpy(),
        "y_final": r.y_final.cpu().numpy(),
        "steps": r.steps.cpu().numpy(),
    }
    if r.features is not None:
        out["features"] = r.features.cpu().numpy()
    if r.y_full is not None:
        out["y"] = r.y_full.cpu().numpy()
    return out


def case_gpu_features(case: Case, y0: np.ndarray, precision: int, rtol: float | None = None, schedule=L.SCHED_QUEUE):
    save = case.save_ts().numpy()
    feats = [(f[0], f[1], f[2]) for f in case.features]
    kw = dict(precision=precision, schedule=schedule, win_begin=case.win_begin(), features=feats)
    t_span = (case.t_span[0], float(save[-1]))
    r = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, t_span, rtol or case.rtol, case.atol, **kw)
    rt = gpu_solve(case.oracle_sys, np.array(case.templates), np.array([case.params]), save, t_span,
                   rtol or case.rtol, case.atol, **kw)
    return r["features"], rt["features"], r


# ---------------------------------------------------------------------------
# trajectories (short, non-chaotic horizon)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("schedule", [L.SCHED_PLAIN, L.SCHED_QUEUE])
@pytest.mark.parametrize("case", [PENDULUM, DUFFING], ids=lambda c: c.name)
def test_fp64_trajectories_match_oracle(case, schedule):
    y0 = seeded_ics(case, 257, seed=3).double().numpy()
    save = np.linspace(0.0, 30.0, 61)
    want = O.solve_batch(case.oracle_sys, y0, np.array([case.params]), save, (0.0, 30.0), 1e-10, 1e-10, keep_full=True)
    got = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, (0.0, 30.0), 1e-10, 1e-10,
                    schedule=schedule, keep_full=True)
    assert (got["status"] == 0).all()
    np.testing.assert_allclose(got["y"], want["y"], rtol=1e-8, atol=1e-9)
    # same algorithm, same control: step counts agree up to a handful of rounding-level decisions
    assert np.abs(got["steps"] - want["steps"]).max() <= 3


def test_mixed_trajectories_track_fp64():
    y0 = seeded_ics(DUFFING, 512, seed=5).double().numpy()
    save = np.linspace(0.0, 30.0, 61)
    # same tolerance on both sides: the difference is FP32 stage rounding plus the
    # step sequence it perturbs, bounded by the accumulated local error (~1e-6/step)
    want = O.solve_batch(O.SYS_DUFFING, y0, np.array([DUFFING.params]), save, (0.0, 30.0), 1e-6, 1e-6, keep_full=True)
    got = gpu_solve(O.SYS_DUFFING, y0, np.array([DUFFING.params]), save, (0.0, 30.0), 1e-6, 1e-6,
                    precision=L.PREC_MIXED, keep_full=True)
    np.testing.assert_allclose(got["y"], want["y"], rtol=1e-3, atol=1e-3)


def test_cross_layout_matches_oracle_expansion():
    y0 = np.array([[0.5, 0.0], [2.0, 1.0], [-1.0, 3.0]])
    P = np.array([[0.1, 0.3, 1.0], [0.1, 0.7, 1.0]])
    save = np.linspace(0.0, 10.0, 21)
    got = gpu_solve(O.SYS_PENDULUM, y0, P, save, (0.0, 10.0), 1e-10, 1e-10, layout=L.LAYOUT_CROSS, keep_full=True)
    idx = np.tile(np.arange(2), 3)
    want = O.solve_batch(O.SYS_PENDULUM, np.repeat(y0, 2, axis=0), P, save, (0.0, 10.0), 1e-10, 1e-10,
                         param_index=idx, keep_full=True)
    np.testing.assert_allclose(got["y"], want["y"], rtol=1e-9, atol=1e-10)


# ---------------------------------------------------------------------------
# fused features over the full horizon
# ---------------------------------------------------------------------------
ALL_FEATS = [(s, k, 0.0) for s in range(2) for k in range(0, 11)] + [(0, 11, 0.0), (1, 11, 0.5), (1, 12, 0.0)]


DENSE = pytest.mark.parametrize("dense", [L.DENSE_INLINE, L.DENSE_DEFERRED], ids=["inline", "deferred"])


@DENSE
@pytest.mark.parametrize("case", [PENDULUM, DUFFING], ids=lambda c: c.name)
def test_all_fused_features_match_oracle(case, dense):
    y0 = seeded_ics(case, 300, seed=11).double().numpy()
    save = case.save_ts().numpy()
    t_span = (0.0, float(save[-1]))
    wb = case.win_begin()
    want = O.solve_batch(case.oracle_sys, y0, np.array([case.params]), save, t_span, 1e-8, 1e-6, win_begin=wb,
                         features=ALL_FEATS)
    got = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, t_span, 1e-8, 1e-6, win_begin=wb,
                    features=ALL_FEATS, dense_mode=dense)
    ok = (got["status"] == 0) & (want["status"] == 0)
    assert ok.all()
    # compare on trajectories whose final states agree (away from basin boundaries)
    # Over t in [0, 1000] two FP64 runs of the same algorithm whose sin/cos differ in the
    # last ulp drift apart by the accumulated global error (~1e-5 relative on the rotating
    # pendulum, whose angle grows to ~2000), so features agree to that level, not to ulps.
    same = np.abs(got["y_final"] - want["y_final"]).max(axis=1) < 1e-5 * (1 + np.abs(want["y_final"]).max(axis=1))
    assert same.mean() > 0.95
    np.testing.assert_allclose(got["features"][same], want["features"][same], rtol=2e-4, atol=1e-6)


@DENSE
@pytest.mark.parametrize("cap", [0, 3])
def test_median_and_crossings_exact_on_identical_windows(dense, cap):
    """Median and crossing counts are order statistics: on short horizons where the
    kernel and oracle windows agree to ~1e-12 they must be equal."""
    y0 = seeded_ics(PENDULUM, 64, seed=2).double().numpy()
    save = np.linspace(0.0, 20.0, 401)
    feats = [(0, 0, 0.0), (1, 0, 0.0), (0, 11, 0.0), (1, 11, 0.25), (1, 11, -0.25)]
    want = O.solve_batch(O.SYS_PENDULUM, y0, np.array([PENDULUM.params]), save, (0.0, 20.0), 1e-10, 1e-10,
                         win_begin=100, features=feats)
    got = gpu_solve(O.SYS_PENDULUM, y0, np.array([PENDULUM.params]), save, (0.0, 20.0), 1e-10, 1e-10,
                    win_begin=100, features=feats, dense_mode=dense, window_record_cap=cap)
    np.testing.assert_allclose(got["features"][:, :2], want["features"][:, :2], rtol=1e-6, atol=1e-7)
    np.testing.assert_array_equal(got["features"][:, 2:], want["features"][:, 2:])


# ---------------------------------------------------------------------------
# golden label fixtures of the reference
# ---------------------------------------------------------------------------
def test_fp64_pendulum_labels_equal_reference_fixture():
    g = np.load(GOLDEN / "labels_pendulum_case1.npz")
    y0 = seeded_ics(PENDULUM, 4000, seed=42).double().numpy()
    f, tf, r = case_gpu_features(PENDULUM, y0, L.PREC_FP64)
    assert (r["status"] == 0).all()
    pred = knn_labels(tf, f)
    assert (pred == g["labels"]).all()
    np.testing.assert_array_equal(np.bincount(pred, minlength=2), g["counts"])


def test_fp64_duffing_labels_match_reference_fixture():
    from sklearn.metrics import matthews_corrcoef

    g = np.load(GOLDEN / "labels_duffing_main.npz")
    y0 = seeded_ics(DUFFING, 4000, seed=42).double().numpy()
    f, tf, _ = case_gpu_features(DUFFING, y0, L.PREC_FP64)
    pred = knn_labels(tf, f)
    assert matthews_corrcoef(g["labels"], pred) >= 0.99
    assert np.abs(np.bincount(pred, minlength=5) - g["counts"]).max() <= 2


@pytest.mark.parametrize("case", [PENDULUM, DUFFING], ids=lambda c: c.name)
def test_mixed_labels_within_delta_bs_of_fp64_oracle(case):
    y0 = seeded_ics(case, 4000, seed=42).double().numpy()
    fo, tfo, _ = oracle_case_features(case, y0)
    want = knn_labels(tfo, fo)
    f, tf, r = case_gpu_features(case, y0, L.PREC_MIXED, rtol=1e-6)
    assert (r["status"] == 0).all()
    got = knn_labels(tf, f)
    k = len(case.templates)
    dbs = np.abs(np.bincount(got, minlength=k) - np.bincount(want, minlength=k)) / len(y0)
    assert dbs.max() <= 0.005
    assert (got == want).mean() >= 0.99


# ---------------------------------------------------------------------------
# device 1-NN labelling
# ---------------------------------------------------------------------------
def test_label_nearest_matches_sklearn():
    rng = np.random.default_rng(0)
    feats = rng.normal(size=(5000, 3))
    feats[7, 1] = np.inf
    feats[9, 0] = np.nan
    tpl = rng.normal(size=(6, 3))
    tpl_cls = np.array([0, 1, 2, 0, 3, 1], dtype=np.int32)
    status = np.zeros(5000, dtype=np.int32)
    status[11] = L.TRAJ_UNBOUNDED
    groups = (np.arange(5000) % 3).astype(np.int32)
    lab, cnt = label_nearest(
        torch.as_tensor(feats, device=DEV),
        torch.as_tensor(tpl, device=DEV),
        torch.as_tensor(tpl_cls, device=DEV),
        4,
        status=torch.as_tensor(status, device=DEV),
        group_of=torch.as_tensor(groups, device=DEV),
        n_groups=3,
    )
    lab = lab.cpu().numpy()
    from sklearn.neighbors import KNeighborsClassifier

    knn = KNeighborsClassifier(n_neighbors=1).fit(impute(tpl), tpl_cls)
    want = knn.predict(impute(feats))
    want[11] = 4
    assert (lab == want).all()
    cnt = cnt.cpu().numpy()
    for g in range(3):
        np.testing.assert_array_equal(cnt[g], np.bincount(want[groups == g], minlength=5))


# ---------------------------------------------------------------------------
# edge cases: ragged sizes, statuses, failure paths
# ---------------------------------------------------------------------------
@DENSE
@pytest.mark.parametrize("n", [1, 31, 33, 4097])
@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
def test_ragged_batch_sizes_queue(n, precision, dense):
    y0 = seeded_ics(PENDULUM, n, seed=9).double().numpy()
    save = np.linspace(0.0, 20.0, 41)
    feats = [(1, 1, 0.0), (0, 5, 0.0)]
    want = O.solve_batch(O.SYS_PENDULUM, y0, np.array([PENDULUM.params]), save, (0, 20), 1e-8, 1e-8, win_begin=20,
                         features=feats)
    if precision == L.PREC_FP64:
        got = gpu_solve(O.SYS_PENDULUM, y0, np.array([PENDULUM.params]), save, (0, 20), 1e-8, 1e-8, win_begin=20,
                        features=feats, precision=precision, grid_blocks=3, block_size=64, dense_mode=dense)
        np.testing.assert_allclose(got["features"], want["features"], rtol=1e-7, atol=1e-7)
    else:
        # FP32 stages at their own tolerance (1e-6) against the oracle at the same tolerance;
        # ICs next to the pendulum's separatrix amplify any perturbation, so a few
        # tenths of a percent of them may leave the 1e-3 band
        want = O.solve_batch(O.SYS_PENDULUM, y0, np.array([PENDULUM.params]), save, (0, 20), 1e-6, 1e-8,
                             win_begin=20, features=feats)
        got = gpu_solve(O.SYS_PENDULUM, y0, np.array([PENDULUM.params]), save, (0, 20), 1e-6, 1e-8, win_begin=20,
                        features=feats, precision=precision, grid_blocks=3, block_size=64, dense_mode=dense)
        close = np.isclose(got["features"], want["features"], rtol=1e-3, atol=1e-3)
        assert close.mean() >= 0.995


def test_status_codes_and_fill():
    save = np.linspace(0.0, 10.0, 11)
    # NaN IC -> non-finite; max_steps=10 -> max_steps
    y0 = np.array([[np.nan, 0.0], [0.1, 0.0]])
    r = gpu_solve(O.SYS_PENDULUM, y0[:1], np.array([PENDULUM.params]), save, (0, 10), 1e-8, 1e-6)
    assert r["status"][0] == L.TRAJ_NONFINITE
    r = gpu_solve(O.SYS_PENDULUM, y0[1:], np.array([PENDULUM.params]), save, (0, 10), 1e-8, 1e-6, max_steps=10)
    assert r["status"][0] == L.TRAJ_MAX_STEPS and r["steps"][0] == 10
    # unbounded event: exponential growth stops, remaining saves are +inf
    r = gpu_solve(O.SYS_LINEAR, np.array([[1.0]]), np.array([[5.0]]), save, (0, 10), 1e-8, 1e-6,
                  unbounded_thr=1e6, keep_full=True, features=[(0, 1, 0.0)])
    want = O.solve_batch(O.SYS_LINEAR, np.array([[1.0]]), np.array([[5.0]]), save, (0, 10), 1e-8, 1e-6,
                         unbounded_thr=1e6, keep_full=True)
    assert r["status"][0] == L.TRAJ_UNBOUNDED
    assert np.isinf(r["y"][-1, 0, 0])
    np.testing.assert_array_equal(np.isinf(r["y"]), np.isinf(want["y"]))
    assert np.isinf(r["features"][0, 0])


def test_huge_initial_condition_does_not_hang():
    save = np.linspace(0.0, 10.0, 11)
    r = gpu_solve(O.SYS_DUFFING, np.array([[1e30, 0.0]]), np.array([DUFFING.params]), save, (0, 10), 1e-8, 1e-6,
                  max_steps=1000)
    assert r["status"][0] in (L.TRAJ_NONFINITE, L.TRAJ_MAX_STEPS, L.TRAJ_DT_UNDERFLOW)


@pytest.mark.parametrize("oracle_sys", [O.SYS_LORENZ, O.SYS_LORENZ_MASKED])
def test_lorenz_variants_match_oracle(oracle_sys):
    rng = np.random.default_rng(1)
    y0 = rng.uniform(-20, 20, size=(128, 3))
    save = np.linspace(0.0, 5.0, 51)
    p = np.array([[10.0, 28.0, 8.0 / 3.0]])
    want = O.solve_batch(oracle_sys, y0, p, save, (0, 5), 1e-10, 1e-10, keep_full=True)
    got = gpu_solve(oracle_sys, y0, p, save, (0, 5), 1e-10, 1e-10, keep_full=True)
    np.testing.assert_allclose(got["y"], want["y"], rtol=1e-6, atol=1e-6)


def test_broken_butterfly_unbounded_labels_match_oracle():
    """Broken-butterfly Lorenz (case_studies/lorenz/setup_lorenz_system.py:28-60): stop at |y|>=200."""
    rng = np.random.default_rng(4)
    y0 = np.stack([rng.uniform(-10, 10, 512), rng.uniform(-20, 20, 512), np.zeros(512)], axis=1)
    save = np.linspace(900.0, 1000.0, 101)
    p = np.array([[0.12, 0.0, -0.6]])
    want = O.solve_batch(O.SYS_LORENZ, y0, p, save, (0, 1000), 1e-8, 1e-6, unbounded_thr=200.0)
    got = gpu_solve(O.SYS_LORENZ, y0, p, save, (0, 1000), 1e-8, 1e-6, unbounded_thr=200.0)
    unb_w = want["status"] == L.TRAJ_UNBOUNDED
    unb_g = got["status"] == L.TRAJ_UNBOUNDED
    assert 0 < unb_w.sum() < len(y0)
    assert (unb_w == unb_g).mean() >= 0.99


# ---------------------------------------------------------------------------
# probed schedule: same steps, same outputs as the queue in processing order
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("case", [PENDULUM, DUFFING], ids=lambda c: c.name)
def test_probed_schedule_is_bit_identical_to_queue(case, precision):
    y0 = seeded_ics(case, 3000, 11).double().numpy()
    save = case.save_ts().numpy()
    feats = [(0, L.FEAT_MAX, 0.0), (0, L.FEAT_STD, 0.0), (1, L.FEAT_MEAN, 0.0), (1, L.FEAT_CROSSINGS, 0.0),
             (0, L.FEAT_MEDIAN, 0.0)]
    kw = dict(precision=precision, win_begin=case.win_begin(), features=feats)
    t_span = (case.t_span[0], float(save[-1]))
    rtol = case.rtol if precision == L.PREC_FP64 else 1e-6
    a = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, t_span, rtol, case.atol,
                  schedule=L.SCHED_QUEUE, **kw)
    for grid in (0, 37):
        b = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, t_span, rtol, case.atol,
                      schedule=L.SCHED_PROBED, grid_blocks=grid, **kw)
        for k in ("status", "steps", "y_final", "features"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_probed_schedule_edge_cases():
    """Stops inside the probe span (unbounded, max_steps, non-finite, bad parameter row),
    record-capacity overflow (redo pass) and a window that starts inside the probe span."""
    rng = np.random.default_rng(5)
    y0 = np.stack([rng.uniform(-10, 10, 700), rng.uniform(-20, 20, 700), np.zeros(700)], axis=1)
    y0[3] = [np.nan, 0.0, 0.0]
    p = np.array([[0.12, 0.0, -0.6], [10.0, 28.0, 8.0 / 3.0]])
    pidx = (np.arange(700) % 2).astype(np.int32)
    pidx[7] = 5  # parameter row out of range
    for save, cap, max_steps in ((np.linspace(900.0, 1000.0, 101), 0, 16**5),
                                 (np.linspace(0.0, 1000.0, 2001), 64, 16**5),
                                 (np.linspace(0.0, 1000.0, 501), 0, 2000)):
        kw = dict(features=[(0, L.FEAT_MEAN, 0.0), (2, L.FEAT_MAX, 0.0)], param_index=pidx,
                  unbounded_thr=200.0, window_record_cap=cap, max_steps=max_steps)
        a = gpu_solve(O.SYS_LORENZ, y0, p, save, (0, 1000), 1e-8, 1e-6, schedule=L.SCHED_QUEUE, **kw)
        b = gpu_solve(O.SYS_LORENZ, y0, p, save, (0, 1000), 1e-8, 1e-6, schedule=L.SCHED_PROBED, **kw)
        for k in ("status", "steps", "y_final", "features"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        st = a["status"]
        assert st[3] == L.TRAJ_NONFINITE and st[7] == L.TRAJ_BAD_INPUT
        assert (st == L.TRAJ_UNBOUNDED).any()
    assert (a["status"] == L.TRAJ_MAX_STEPS).any()


# the wider feature set: streaming kinds (from the running sums) and window kinds
# (second pass over the stored FP32 window), on one state
WIDE_FEATS = [(0, k, 0.0) for k in (L.FEAT_SUM, L.FEAT_ABS_ENERGY, L.FEAT_LENGTH, L.FEAT_VARIATION_COEFF)] + [
    (0, L.FEAT_QUANTILE, 0.1), (0, L.FEAT_QUANTILE, 0.75), (0, L.FEAT_KURTOSIS, 0.0), (0, L.FEAT_SKEWNESS, 0.0),
    (0, L.FEAT_ABS_SUM_CHANGES, 0.0), (0, L.FEAT_MEAN_ABS_CHANGE, 0.0), (0, L.FEAT_MEAN_CHANGE, 0.0),
    (0, L.FEAT_MEAN_SECOND_DERIV, 0.0), (0, L.FEAT_COUNT_ABOVE_MEAN, 0.0), (0, L.FEAT_COUNT_BELOW_MEAN, 0.0),
    (0, L.FEAT_COUNT_ABOVE, 0.0), (0, L.FEAT_COUNT_BELOW, 0.5), (0, L.FEAT_NUMBER_PEAKS, 1.0),
    (0, L.FEAT_NUMBER_PEAKS, 3.0), (0, L.FEAT_AUTOCORRELATION, 1.0), (0, L.FEAT_AUTOCORRELATION, 7.0),
    (0, L.FEAT_RATIO_BEYOND_R_SIGMA, 1.0), (0, L.FEAT_MEDIAN, 0.0),
]
COUNT_KINDS = {L.FEAT_COUNT_ABOVE_MEAN, L.FEAT_COUNT_BELOW_MEAN, L.FEAT_NUMBER_PEAKS}
FRACTION_KINDS = {L.FEAT_COUNT_ABOVE, L.FEAT_COUNT_BELOW, L.FEAT_RATIO_BEYOND_R_SIGMA}


@DENSE
@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
def test_wider_feature_set_matches_oracle(dense, precision):
    """Short horizon (t in [0, 30], window [20, 30] x 500 saves) where kernel and oracle
    trajectories agree to ~1e-8 (FP64) / ~1e-5 (mixed): continuous features to 2e-4
    relative (the window kinds read FP32-stored samples); counts and fractions to a
    sample or two (a sample within rounding of the mean or level may flip)."""
    case = DUFFING
    y0 = seeded_ics(case, 200, seed=13).double().numpy()
    save = np.asarray(torch.linspace(0.0, 30.0, 1501, dtype=torch.float32).double())
    wb = int(np.nonzero(save >= 20.0)[0][0])
    n = len(save) - wb
    rtol = case.rtol if precision == L.PREC_FP64 else 1e-6
    want = O.solve_batch(case.oracle_sys, y0, np.array([case.params]), save, (0.0, 30.0), 1e-10, 1e-10,
                         win_begin=wb, features=WIDE_FEATS)
    got = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, (0.0, 30.0), min(rtol, 1e-8), 1e-10,
                    win_begin=wb, features=WIDE_FEATS, dense_mode=dense, precision=precision)
    assert (got["status"] == 0).all()
    g, w = got["features"], want["features"]
    for c, (_, kind, _) in enumerate(WIDE_FEATS):
        if kind in COUNT_KINDS:
            assert np.abs(g[:, c] - w[:, c]).max() <= 2, (c, kind)
        elif kind in FRACTION_KINDS:
            assert np.abs(g[:, c] - w[:, c]).max() <= 2.0 / n, (c, kind)
        else:
            tol = 2e-4 if precision == L.PREC_FP64 else 2e-3
            scale = np.abs(w[:, c]).max() + 1e-12
            np.testing.assert_allclose(g[:, c], w[:, c], rtol=tol, atol=tol * 1e-3 * scale, err_msg=f"col {c} kind {kind}")


MORE_FEATS = [(0, k, float(c)) for k in (L.FEAT_FFT_REAL, L.FEAT_FFT_IMAG, L.FEAT_FFT_ANGLE) for c in (1, 250)] + [
    (0, L.FEAT_FFT_ABS, 1.0), (0, L.FEAT_FFT_ABS, 250.0),
    (0, L.FEAT_FFT_ABS, 0.0), (0, L.FEAT_FFT_REAL, 251.0),
    (0, L.FEAT_TREND_SLOPE, 0.0), (0, L.FEAT_TREND_INTERCEPT, 0.0), (0, L.FEAT_TREND_RVALUE, 0.0),
    (0, L.FEAT_TREND_PVALUE, 0.0), (0, L.FEAT_TREND_STDERR, 0.0),
    (1, L.FEAT_FIRST_LOC_MAX, 0.0), (1, L.FEAT_FIRST_LOC_MIN, 0.0), (1, L.FEAT_LAST_LOC_MAX, 0.0),
    (1, L.FEAT_LAST_LOC_MIN, 0.0), (0, L.FEAT_CID_CE, 1.0), (0, L.FEAT_CID_CE, 0.0), (0, L.FEAT_C3, 2.0),
    (0, L.FEAT_C3, 300.0), (1, L.FEAT_TIME_REVERSAL, 3.0),
    (0, L.FEAT_SPKT_WELCH, 5.0), (0, L.FEAT_LARGE_STD, 0.25), (1, L.FEAT_SYMMETRY_LOOKING, 0.1),
    (0, L.FEAT_INDEX_MASS_QUANTILE, 0.5), (0, L.FEAT_LONGEST_STRIKE_ABOVE, 0.0),
    (1, L.FEAT_LONGEST_STRIKE_BELOW, 0.0),
]
# fourth group (the window pass takes at most 32 columns per call)
EXTRA_FEATS = [(0, L.FEAT_HAS_DUP_MAX, 0.0), (1, L.FEAT_HAS_DUP_MIN, 0.0), (0, L.FEAT_BINNED_ENTROPY, 10.0),
               (1, L.FEAT_BINNED_ENTROPY, 37.0), (0, L.FEAT_MEAN_N_ABS_MAX, 1.0), (0, L.FEAT_MEAN_N_ABS_MAX, 7.0),
               (0, L.FEAT_BENFORD, 0.0), (1, L.FEAT_BENFORD, 0.0)]
LOCATION_KINDS = {L.FEAT_FIRST_LOC_MAX, L.FEAT_FIRST_LOC_MIN, L.FEAT_LAST_LOC_MAX, L.FEAT_LAST_LOC_MIN,
                  L.FEAT_INDEX_MASS_QUANTILE}
FLAG_KINDS = {L.FEAT_LARGE_STD, L.FEAT_SYMMETRY_LOOKING, L.FEAT_HAS_DUP_MAX, L.FEAT_HAS_DUP_MIN}  # 1 / 0 decisions
RUN_KINDS = {L.FEAT_LONGEST_STRIKE_ABOVE, L.FEAT_LONGEST_STRIKE_BELOW}


@DENSE
@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
def test_frequency_trend_location_features_match_oracle(dense, precision):
    """FFT coefficients, linear trend, extreme locations, cid_ce, c3 and the time
    reversal statistic from the window pass against the oracle (the short horizon
    of the wider-set test): continuous features to 2e-4 relative (2e-3 mixed); the
    location of an extreme within 2 samples (FP64) / 10 samples (mixed) of the
    oracle's, since a flat extremum moves with the trajectory's last digits.  The
    window pass reads FP32-stored samples, so a DFT coefficient carries up to
    2^-24 * sum |x_n| (about 3e-5 here) of absolute error whatever its size: real,
    imaginary part and magnitude get that absolute tolerance, and an angle is
    compared on the unit circle where the magnitude resolves it."""
    case = DUFFING
    y0 = seeded_ics(case, 200, seed=13).double().numpy()
    save = np.asarray(torch.linspace(0.0, 30.0, 1501, dtype=torch.float32).double())
    wb = int(np.nonzero(save >= 20.0)[0][0])
    n = len(save) - wb
    rtol = case.rtol if precision == L.PREC_FP64 else 1e-6
    want = O.solve_batch(case.oracle_sys, y0, np.array([case.params]), save, (0.0, 30.0), min(rtol, 1e-8), 1e-10,
                         win_begin=wb, features=MORE_FEATS)
    got = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, (0.0, 30.0), min(rtol, 1e-8), 1e-10,
                    win_begin=wb, features=MORE_FEATS, dense_mode=dense, precision=precision)
    assert (got["status"] == 0).all()
    g, w = got["features"], want["features"]
    fft_atol = 3e-5 if precision == L.PREC_FP64 else 3e-3
    abs_col = {prm: c for c, (_, kind, prm) in enumerate(MORE_FEATS) if kind == L.FEAT_FFT_ABS}
    for c, (_, kind, prm) in enumerate(MORE_FEATS):
        if kind == L.FEAT_FFT_ANGLE:
            mag = w[:, abs_col[prm]]
            keep = mag > 100 * fft_atol
            chord = np.abs(np.exp(1j * g[keep, c]) - np.exp(1j * w[keep, c]))
            assert chord.max(initial=0.0) <= 2e-2, (c, kind, prm)  # angle error <= fft_atol / |X| <= 1e-2
        elif kind in (L.FEAT_FFT_REAL, L.FEAT_FFT_IMAG, L.FEAT_FFT_ABS) and prm != 251.0:
            np.testing.assert_allclose(g[:, c], w[:, c], rtol=2e-4, atol=fft_atol, err_msg=f"col {c} kind {kind}")
        elif kind in LOCATION_KINDS:
            lim = (2.0 if precision == L.PREC_FP64 else 10.0) / n
            assert np.abs(g[:, c] - w[:, c]).max() <= lim + 1e-12, (c, kind)
        elif kind in FLAG_KINDS:  # a value within rounding of its threshold may flip
            assert (g[:, c] != w[:, c]).sum() <= 2, (c, kind)
        elif kind in RUN_KINDS:  # a sample within rounding of the mean may end a run
            assert (g[:, c] != w[:, c]).mean() <= 0.05, (c, kind)
        elif kind == L.FEAT_SPKT_WELCH:
            np.testing.assert_allclose(g[:, c], w[:, c], rtol=2e-3, atol=fft_atol * 2e-2, err_msg=f"col {c}")
        elif kind == L.FEAT_FFT_REAL and prm == 251.0 or kind == L.FEAT_C3 and prm == 300.0:
            assert (g[:, c] == 0.0).all() and (w[:, c] == 0.0).all()  # past the last coefficient / lag
        else:
            tol = 2e-4 if precision == L.PREC_FP64 else 2e-3
            scale = np.abs(w[:, c]).max() + 1e-12
            np.testing.assert_allclose(g[:, c], w[:, c], rtol=tol, atol=tol * 1e-2 * scale,
                                       err_msg=f"col {c} kind {kind}")


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
def test_entropy_duplicate_benford_features_match_oracle(precision):
    """Binned entropy, duplicate extremes, mean of the n largest |x| and the Benford
    correlation from the window pass against the oracle (the short horizon of the
    wider-set test).  Bin and first-digit counts can move by a sample whose value
    sits within rounding of a bin edge or a power of ten, so entropy and Benford
    compare to 1e-2; the duplicate flags are exact decisions on FP32-stored
    samples (the oracle's FP64 trajectory rarely repeats a value)."""
    case = DUFFING
    y0 = seeded_ics(case, 200, seed=13).double().numpy()
    save = np.asarray(torch.linspace(0.0, 30.0, 1501, dtype=torch.float32).double())
    wb = int(np.nonzero(save >= 20.0)[0][0])
    rtol = case.rtol if precision == L.PREC_FP64 else 1e-6
    want = O.solve_batch(case.oracle_sys, y0, np.array([case.params]), save, (0.0, 30.0), min(rtol, 1e-8), 1e-10,
                         win_begin=wb, features=EXTRA_FEATS)
    got = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, (0.0, 30.0), min(rtol, 1e-8), 1e-10,
                    win_begin=wb, features=EXTRA_FEATS, precision=precision)
    assert (got["status"] == 0).all()
    g, w = got["features"], want["features"]
    for c, (_, kind, _) in enumerate(EXTRA_FEATS):
        if kind in (L.FEAT_HAS_DUP_MAX, L.FEAT_HAS_DUP_MIN):
            assert set(np.unique(g[:, c])) <= {0.0, 1.0}
            assert (g[:, c] != w[:, c]).mean() <= 0.1, (c, kind)
        elif kind == L.FEAT_MEAN_N_ABS_MAX:
            np.testing.assert_allclose(g[:, c], w[:, c], rtol=2e-4 if precision == L.PREC_FP64 else 2e-3)
        else:
            np.testing.assert_allclose(g[:, c], w[:, c], rtol=1e-2, atol=1e-2, err_msg=f"col {c} kind {kind}")


SORTED_FEATS = [(0, L.FEAT_HAS_DUPLICATE, 0.0), (0, L.FEAT_PCT_REOCCURRING_POINTS, 0.0),
                (0, L.FEAT_PCT_REOCCURRING_VALUES, 0.0), (0, L.FEAT_SUM_REOCCURRING_POINTS, 0.0),
                (0, L.FEAT_SUM_REOCCURRING_VALUES, 0.0), (0, L.FEAT_RATIO_UNIQUE_VALUES, 0.0),
                (0, L.FEAT_VAR_LARGER_THAN_STD, 0.0), (0, L.FEAT_COUNT_VALUE, 0.0)]


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("n_save", [2001, 20001])
def test_repeated_value_features_on_identical_windows(precision, n_save):
    """Duplicate and reoccurrence features from the sorted window pass against the
    oracle evaluated on the kernel's own FP32 window (the save points written to
    y_full are the samples the window holds, rounded to FP32 alike), so counts and
    ratios must agree exactly and the sums to FP64 summation order.  Exponential
    decay at four rates under relative error control: the slow one keeps distinct
    normal floats (no repeats), the fast ones reach FP32 subnormals and then zero,
    where values repeat in long runs.  20,001 saves put 16,001 samples in the window: a 64 KB sort in shared
    memory."""
    rng = np.random.default_rng(5)
    n = 64
    y0 = rng.uniform(0.5, 2.0, size=(n, 1))
    rates = np.array([[-0.3], [-0.9], [-1.0], [-1.1]])
    pidx = np.arange(n, dtype=np.int32) % 4
    save = np.linspace(90.0, 140.0, n_save)
    wb = int(np.nonzero(save >= 100.0)[0][0])
    # relative error control all the way down (FP64: atol 0; the FP32 stages of the
    # mixed kernel need a nonzero atol once the state underflows)
    atol = 0.0 if precision == L.PREC_FP64 else 1e-30
    got = gpu_solve(O.SYS_LINEAR, y0, rates, save, (0.0, 140.0), 1e-8, atol, precision=precision,
                    win_begin=wb, features=SORTED_FEATS, param_index=pidx, keep_full=True)
    assert (got["status"] == 0).all()
    win = got["y"][wb:, :, 0].astype(np.float32).astype(np.float64)  # (n_win, n)
    want = np.array([[O.window_feature(k, p, win[:, j]) for (_, k, p) in SORTED_FEATS] for j in range(n)])
    g = got["features"]
    sums = [c for c, (_, k, _) in enumerate(SORTED_FEATS)
            if k in (L.FEAT_SUM_REOCCURRING_POINTS, L.FEAT_SUM_REOCCURRING_VALUES)]
    exact = [c for c in range(len(SORTED_FEATS)) if c not in sums]
    np.testing.assert_array_equal(g[:, exact], want[:, exact])
    np.testing.assert_allclose(g[:, sums], want[:, sums], rtol=1e-12, atol=1e-300)
    dup = g[:, 0]
    # both regimes present (the mixed kernel's FP32 state settles into absolute-
    # tolerance noise rather than underflowing, so fewer of its windows repeat)
    assert (dup[pidx == 0] == 0.0).all()
    assert (dup[pidx > 0] == 1.0).sum() >= (n // 4 if precision == L.PREC_FP64 else 1)


ACF_PAIR_FEATS = [(0, L.FEAT_PARTIAL_AUTOCORRELATION, 1.0), (0, L.FEAT_PARTIAL_AUTOCORRELATION, 7.0),
                  (1, L.FEAT_PARTIAL_AUTOCORRELATION, 63.0), (0, L.FEAT_PARTIAL_AUTOCORRELATION, 0.0),
                  (0, L.FEAT_AGG_AUTOCORR_MEAN, 40.0), (1, L.FEAT_AGG_AUTOCORR_MEDIAN, 40.0),
                  (0, L.FEAT_AGG_AUTOCORR_MEDIAN, 7.0), (1, L.FEAT_AGG_AUTOCORR_VAR, 128.0),
                  (0, L.FEAT_ENERGY_RATIO_BY_CHUNKS, 10.0, 0.0), (1, L.FEAT_ENERGY_RATIO_BY_CHUNKS, 10.0, 9.0),
                  (0, L.FEAT_ENERGY_RATIO_BY_CHUNKS, 3.0, 5.0), (0, L.FEAT_COUNT_IN_RANGE, -1.0, 1.0),
                  (1, L.FEAT_COUNT_IN_RANGE, 0.0, 1e12), (0, L.FEAT_CHANGE_QUANTILES_MEAN, 0.2, 0.8),
                  (1, L.FEAT_CHANGE_QUANTILES_VAR, 0.0, 0.4), (0, L.FEAT_CHANGE_QUANTILES_ABS_MEAN, 0.4, 1.0),
                  (1, L.FEAT_CHANGE_QUANTILES_ABS_VAR, 0.2, 0.8), (0, L.FEAT_CHANGE_QUANTILES_VAR, 0.5, 0.5),
                  (0, L.FEAT_ACF_PERIOD_STRENGTH, 2.0, 0.3), (0, L.FEAT_ACF_PERIOD_LAG, 2.0, 0.3),
                  (1, L.FEAT_ACF_PERIOD_LAG, 50.0, 0.5), (1, L.FEAT_ACF_PERIOD_STRENGTH, 2.0, 0.99)]
# second group (a solve takes at most 32 columns)
DYN_FEATS = [(0, L.FEAT_AGG_TREND_MEAN, 50.0, 0.0), (1, L.FEAT_AGG_TREND_VAR, 5.0, 2.0),
                  (0, L.FEAT_AGG_TREND_MIN, 20.0, 4.0), (1, L.FEAT_AGG_TREND_MAX, 200.0, 3.0),
                  (0, L.FEAT_AGG_TREND_MEAN, 400.0, 1.0), (0, L.FEAT_AR_COEFFICIENT, 10.0, 0.0),
                  (1, L.FEAT_AR_COEFFICIENT, 10.0, 9.0), (0, L.FEAT_AR_COEFFICIENT, 4.0, 2.0),
                  (1, L.FEAT_AR_COEFFICIENT, 3.0, 3.0), (0, L.FEAT_CWT, 5.0, 100.0), (1, L.FEAT_CWT, 20.0, 0.0),
                  (0, L.FEAT_CWT, 2.0, 3.0), (1, L.FEAT_CWT, 10.0, -1.0), (0, L.FEAT_CWT, 200.0, 700.0),
                  (0, L.FEAT_FRIEDRICH, 3.0, 0.0), (1, L.FEAT_FRIEDRICH, 3.0, 3.0), (0, L.FEAT_FRIEDRICH, 1.0, 1.0),
                  (0, L.FEAT_LANGEVIN, 3.0, 0.0), (1, L.FEAT_LANGEVIN, 1.0, 0.0),
                  (0, L.FEAT_ADF_TESTSTAT, 0.0, 0.0), (1, L.FEAT_ADF_PVALUE, 0.0, 0.0),
                  (0, L.FEAT_ADF_USEDLAG, 0.0, 0.0), (0, L.FEAT_NUMBER_CWT_PEAKS, 1.0, 0.0),
                  (1, L.FEAT_NUMBER_CWT_PEAKS, 5.0, 0.0), (0, L.FEAT_NUMBER_CWT_PEAKS, 64.0, 0.0)]


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
def test_acf_and_two_parameter_features_on_identical_windows(precision):
    """Partial and aggregated autocorrelation, autocorrelation periodicity, chunk
    energy ratio, count in range, change quantiles, trends of chunk aggregates,
    AR, Ricker-wavelet and Friedrich coefficients, the Langevin fixed point,
    augmented Dickey-Fuller and CWT-peak counts from the window pass against the oracle evaluated on the
    kernel's own FP32 window (y_full holds the samples the window stores).  Counts
    and periods are exact; the rest differ by summation order only: the
    autocorrelations (at most 1 in size) to 1e-10 absolute, the others to 1e-9
    relative; AR coefficients solve a Toeplitz system of autocorrelations near 1
    (condition ~1e6 through the 1e-6 ridge): 1e-6 relative."""
    y0 = seeded_ics(DUFFING, 96, seed=21).double().numpy()
    save = np.linspace(0.0, 40.0, 2001)
    wb = int(np.nonzero(save >= 25.0)[0][0])
    for feats in (ACF_PAIR_FEATS, DYN_FEATS):
        g = _check_identical_windows(y0, save, wb, precision, feats)
        if feats is ACF_PAIR_FEATS:
            assert (g[:, 3] == 1.0).all()  # lag 0
            assert np.ptp(g[:, 11]) > 0 and (g[:, 13] != 0).any()  # non-trivial counts and corridors
            assert (g[:, 19] > 0).mean() > 0.5  # most windows of the forced oscillation show a period


def _check_identical_windows(y0, save, wb, precision, feats):
    got = gpu_solve(O.SYS_DUFFING, y0, np.array([DUFFING.params]), save, (0.0, float(save[-1])), 1e-8, 1e-10,
                    precision=precision, win_begin=wb, features=feats, keep_full=True)
    assert (got["status"] == 0).all()
    win = got["y"][wb:].astype(np.float32).astype(np.float64)  # (n_win, n, 2)
    want = np.array([[O.window_feature(f[1], f[2], win[:, j, f[0]], f[3] if len(f) > 3 else 0.0)
                      for f in feats] for j in range(len(y0))])
    g = got["features"]
    for c, f in enumerate(feats):
        if L.FEAT_PARTIAL_AUTOCORRELATION <= f[1] <= L.FEAT_AGG_AUTOCORR_VAR or f[1] == L.FEAT_ACF_PERIOD_STRENGTH:
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=0.0, atol=1e-10, err_msg=f"col {c} {f}")
        elif f[1] == L.FEAT_LANGEVIN:  # a window value chosen by the sign of a fit: equal or a near-zero flip
            assert (g[:, c] == want[:, c]).mean() >= 0.95, (c, f)
        elif f[1] in (L.FEAT_AR_COEFFICIENT, L.FEAT_FRIEDRICH):  # normal equations: ill-conditioned
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-6, atol=1e-9, err_msg=f"col {c} {f}")
        elif f[1] in (L.FEAT_COUNT_IN_RANGE, L.FEAT_ACF_PERIOD_LAG, L.FEAT_NUMBER_CWT_PEAKS, L.FEAT_ADF_USEDLAG):
            np.testing.assert_array_equal(g[:, c], want[:, c], err_msg=f"col {c} {f}")
        else:
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-9, atol=1e-15, err_msg=f"col {c} {f}")
    return g


def test_two_parameter_features_through_the_extractor_names():
    """FCParameters entries with several parameters (the reference's settings,
    ts_torch/settings.py:263-346) become one fused column each, in config order."""
    from pybasin_b200 import B200Dopri5Solver, DuffingODE, FusedFeatureExtractor

    cfg = {"agg_autocorrelation": [{"f_agg": s, "maxlag": 40} for s in ("mean", "median", "var")],
           "partial_autocorrelation": [{"lag": 2}],
           "change_quantiles": [{"ql": 0.2, "qh": 0.8, "isabs": True, "f_agg": "mean"}],
           "count_in_range": [{"min_val": -1, "max_val": 1}],
           "energy_ratio_by_chunks": [{"num_segments": 10, "segment_focus": i} for i in range(10)],
           "autocorrelation_periodicity": [{"output": "strength"}, {"output": "period"}],
           "spectral_frequency_ratio": None, "fft_aggregated": [{"aggtype": "kurtosis"}],
           "agg_linear_trend": [{"attr": "rvalue", "chunk_size": 50, "f_agg": "max"}],
           "ar_coefficient": [{"coeff": 1, "k": 10}], "linear_trend_timewise": [{"attr": "slope"}],
           "cwt_coefficients": [{"widths": (5,), "coeff": 3, "w": 5}], "friedrich_coefficients": None,
           "max_langevin_fixed_point": None, "augmented_dickey_fuller": [{"attr": "pvalue"}],
           "number_cwt_peaks": [{"max_width": 5}]}
    fx = FusedFeatureExtractor(time_steady=900.0, features=None, features_per_state={0: cfg}, normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=2000, t_eval=(900, 1000), device="cuda:0",
                              precision="fp64", feature_extractor=fx)
    y0 = seeded_ics(DUFFING, 32, seed=3).double()
    t, y = solver.integrate(DuffingODE(dict(zip(("delta", "k3", "A"), DUFFING.params))), y0)
    f = fx.extract_features(type("S", (), {"y": y})())
    assert f.shape == (32, 28) and torch.isfinite(f).all()
    assert fx.feature_names[0] == "state_0__agg_autocorrelation__f_agg_mean__maxlag_40"
    assert fx.feature_names[19] == "state_0__fft_aggregated__aggtype_kurtosis"
    assert fx.feature_names[22] == "state_0__linear_trend_timewise__attr_slope"
    # the ten chunk energy ratios partition the window's energy (200 samples per chunk)
    np.testing.assert_allclose(f[:, 6:16].sum(dim=1).cpu().numpy(), 1.0, rtol=1e-9)


SPECTRAL_FEATS = [(0, L.FEAT_SPECTRAL_FREQ_RATIO, 0.0), (1, L.FEAT_SPECTRAL_FREQ_RATIO, 0.0),
                  (0, L.FEAT_FFT_AGG_CENTROID, 0.0), (1, L.FEAT_FFT_AGG_VARIANCE, 0.0),
                  (0, L.FEAT_FFT_AGG_SKEW, 0.0), (1, L.FEAT_FFT_AGG_KURTOSIS, 0.0)]


@pytest.mark.parametrize("n_save", [2001, 2002])
def test_spectral_features_on_identical_windows(n_save):
    """spectral_frequency_ratio and fft_aggregated from the spectrum pass (FP64
    Goertzel recurrences) against the oracle's direct DFT on the kernel's own FP32
    window, odd and even window lengths: the spectrum moments to 1e-8 relative; the
    frequency ratio picks bins by rank, so it is equal wherever the competing bins'
    powers differ by more than the two methods' rounding (all but a few windows)."""
    y0 = seeded_ics(DUFFING, 128, seed=23).double().numpy()
    save = np.linspace(0.0, 60.0, n_save)
    wb = int(np.nonzero(save >= 20.0)[0][0])
    got = gpu_solve(O.SYS_DUFFING, y0, np.array([DUFFING.params]), save, (0.0, 60.0), 1e-8, 1e-10,
                    win_begin=wb, features=SPECTRAL_FEATS, keep_full=True)
    assert (got["status"] == 0).all()
    win = got["y"][wb:].astype(np.float32).astype(np.float64)
    want = np.array([[O.window_feature(k, p, win[:, j, st]) for (st, k, p) in SPECTRAL_FEATS] for j in range(len(y0))])
    g = got["features"]
    for c, (_, k, _) in enumerate(SPECTRAL_FEATS):
        if k == L.FEAT_SPECTRAL_FREQ_RATIO:
            assert (g[:, c] == want[:, c]).mean() >= 0.97, c
            assert (g[:, c] > 0).all()
        else:
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-8, atol=1e-12, err_msg=f"col {c}")


SYMBOLIC_FEATS = [(0, L.FEAT_PERMUTATION_ENTROPY, 1.0, 3.0), (1, L.FEAT_PERMUTATION_ENTROPY, 2.0, 5.0),
                  (0, L.FEAT_PERMUTATION_ENTROPY, 1.0, 7.0), (1, L.FEAT_PERMUTATION_ENTROPY, 40.0, 4.0),
                  (0, L.FEAT_LEMPEL_ZIV, 2.0), (1, L.FEAT_LEMPEL_ZIV, 10.0), (0, L.FEAT_LEMPEL_ZIV, 100.0),
                  (1, L.FEAT_LEMPEL_ZIV, 255.0), (0, L.FEAT_CORR_DIM, 4.0, 1 * 1024 + 50.0),
                  (1, L.FEAT_CORR_DIM, 2.0, 3 * 1024 + 20.0), (0, L.FEAT_LYAP_R, 10 * 1024 + 20.0, 1.0),
                  (1, L.FEAT_LYAP_R, 4 * 1024 + 10.0, 2.0), (0, L.FEAT_FOURIER_ENTROPY, 10.0)]


@pytest.mark.parametrize("n_save", [1001, 8191 + 250])
def test_entropy_and_complexity_features_on_identical_windows(n_save):
    """Permutation entropy, Lempel-Ziv complexity, correlation dimension, the
    largest Lyapunov exponent and Fourier entropy from the symbolic and spectrum
    passes against the oracle on the kernel's own FP32
    window: the phrase counts exactly, the permutation entropy to summation order,
    the Fourier entropy to 1e-8 (the spectrum pass's rounding).  The
    long case fills the largest Lempel-Ziv window (8,191 samples; a 128 KB trie
    table)."""
    y0 = seeded_ics(DUFFING, 64, seed=29).double().numpy()
    save = np.linspace(0.0, 60.0, n_save)
    wb = 250 if n_save > 8191 else int(np.nonzero(save >= 20.0)[0][0])
    # the oracle's direct DFT and pair counts are O(n^2): the long case keeps the linear kinds
    feats = SYMBOLIC_FEATS if n_save < 8191 else [f for f in SYMBOLIC_FEATS
                                                  if f[1] not in (L.FEAT_FOURIER_ENTROPY, L.FEAT_CORR_DIM,
                                                                  L.FEAT_LYAP_R)]
    got = gpu_solve(O.SYS_DUFFING, y0, np.array([DUFFING.params]), save, (0.0, 60.0), 1e-8, 1e-10,
                    win_begin=wb, features=feats, keep_full=True)
    assert (got["status"] == 0).all()
    win = got["y"][wb:].astype(np.float32).astype(np.float64)
    want = np.array([[O.window_feature(f[1], f[2], win[:, j, f[0]], f[3] if len(f) > 3 else 0.0) for f in feats]
                     for j in range(len(y0))])
    g = got["features"]
    for c, f in enumerate(feats):
        if f[1] == L.FEAT_LEMPEL_ZIV:
            np.testing.assert_array_equal(g[:, c], want[:, c], err_msg=f"col {c} {f}")
        elif f[1] == L.FEAT_LYAP_R:  # same neighbours; divergences rounded to FP32 as the reference stores them
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-5, atol=1e-7, err_msg=f"col {c} {f}")
        elif f[1] == L.FEAT_CORR_DIM:  # exact pair counts; the log-log fit to summation order
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-9, atol=1e-12, err_msg=f"col {c} {f}")
        elif f[1] == L.FEAT_FOURIER_ENTROPY:  # spectrum by Goertzel: rounding grows as n eps / sin(w)
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-8, atol=1e-12, err_msg=f"col {c} {f}")
        else:
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-11, atol=1e-14, err_msg=f"col {c} {f}")
    assert (g[:, 4] > 0).all() and (g[:, 0] > 0).all()


@pytest.mark.parametrize("n_save", [3001, 4800])
def test_pair_count_features_on_long_windows(n_save):
    """correlation_dimension and lyapunov_r are O(n^2) per column (all pairs of
    delay vectors; every vector's nearest neighbour): on windows of a few thousand
    samples, a handful of trajectories, against the oracle on the kernel's own FP32
    window, with the symbolic pass's time per (trajectory, column) printed."""
    y0 = seeded_ics(DUFFING, 6, seed=31).double().numpy()
    save = np.linspace(0.0, 160.0, n_save)
    wb = n_save // 10
    feats = [(0, L.FEAT_CORR_DIM, 4.0, 2 * 1024 + 50.0), (1, L.FEAT_CORR_DIM, 2.0, 1 * 1024 + 20.0),
             (0, L.FEAT_LYAP_R, 10 * 1024 + 20.0, 1.0), (1, L.FEAT_LYAP_R, 4 * 1024 + 10.0, 2.0)]
    got = gpu_solve(O.SYS_DUFFING, y0, np.array([DUFFING.params]), save, (0.0, 160.0), 1e-8, 1e-10,
                    win_begin=wb, features=feats, keep_full=True)
    assert (got["status"] == 0).all()
    win = got["y"][wb:].astype(np.float32).astype(np.float64)
    want = np.array([[O.window_feature(f[1], f[2], win[:, j, f[0]], f[3]) for f in feats] for j in range(len(y0))])
    g = got["features"]
    for c, f in enumerate(feats):
        if f[1] == L.FEAT_LYAP_R:
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-5, atol=1e-7, err_msg=f"col {c} {f}")
        else:
            np.testing.assert_allclose(g[:, c], want[:, c], rtol=1e-9, atol=1e-12, err_msg=f"col {c} {f}")
    # cost of the pass: the same solve with and without the pair-count columns
    def timed(columns):
        ts = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            gpu_solve(O.SYS_DUFFING, y0, np.array([DUFFING.params]), save, (0.0, 160.0), 1e-8, 1e-10,
                      win_begin=wb, features=columns)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return min(ts)

    extra = timed(feats) - timed([(0, L.FEAT_MEDIAN, 0.0)])
    print(f"pair-count pass, window {n_save - wb}: {extra / (len(y0) * len(feats)):.3f} ms per (trajectory, column)")


def test_spectral_features_reject_oversized_windows():
    """The spectrum sits in shared memory: more than 16,384 window samples is refused."""
    save = np.linspace(0.0, 1.0, L.SPECTRAL_WINDOW_MAX + 1)
    with pytest.raises(RuntimeError, match="unsupported"):
        gpu_solve(O.SYS_LINEAR, np.ones((2, 1)), np.array([[-1.0]]), save, (0.0, 1.0), 1e-6, 1e-9,
                  win_begin=0, features=[(0, L.FEAT_FFT_AGG_CENTROID, 0.0)])


def test_sorted_window_features_reject_oversized_windows():
    """The sorted kinds hold the window in shared memory: more than 32,768 window
    samples is refused before any launch."""
    save = np.linspace(0.0, 1.0, L.SORTED_WINDOW_MAX + 2)
    with pytest.raises(RuntimeError, match="unsupported"):
        gpu_solve(O.SYS_LINEAR, np.ones((2, 1)), np.array([[-1.0]]), save, (0.0, 1.0), 1e-6, 1e-9,
                  win_begin=0, features=[(0, L.FEAT_HAS_DUPLICATE, 0.0)])


def test_wider_features_through_the_extractor_names():
    """FCParameters names and parameters as in the reference's settings (ts_torch/settings.py:223-355)."""
    from pybasin_b200 import B200Dopri5Solver, DuffingODE, FusedFeatureExtractor

    cfg = {"quantile": [{"q": 0.1}, {"q": 0.9}], "kurtosis": None, "number_peaks": [{"n": 1}, {"n": 3}],
           "autocorrelation": [{"lag": 2}], "count_above": [{"t": 0}], "sum_values": None}
    fx = FusedFeatureExtractor(time_steady=900.0, features=None, features_per_state={0: cfg}, normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=2000, t_eval=(900, 1000), device="cuda:0",
                              precision="fp64", feature_extractor=fx)
    y0 = seeded_ics(DUFFING, 64, seed=3).double()
    t, y = solver.integrate(DuffingODE(dict(zip(("delta", "k3", "A"), DUFFING.params))), y0)
    f = fx.extract_features(type("S", (), {"y": y})())
    assert f.shape == (64, 8) and torch.isfinite(f).all()
    names = fx.feature_names
    assert names[0] == "state_0__quantile__q_0.1" and "state_0__number_peaks__n_3" in names
    # ordering sanity: quantile 0.1 <= quantile 0.9 on every trajectory
    assert (f[:, 0] <= f[:, 1]).all()


def test_orbit_data_peaks_match_oracle_trajectories():
    """Orbit-diagram peaks (src/pybasin/utils.py:254-303) from the solve vs strict local
    maxima of the oracle's sampled window (short horizon: FP64 trajectories agree to ~1e-8)."""
    from pybasin_b200 import B200Dopri5Solver, DuffingODE

    y0 = seeded_ics(DUFFING, 48, seed=21).double()
    solver = B200Dopri5Solver(t_span=(0, 60), t_steps=1201, device="cuda:0", rtol=1e-10, atol=1e-10,
                              precision="fp64")
    od = solver.orbit_data(DuffingODE(dict(zip(("delta", "k3", "A"), DUFFING.params))), y0, dof=[0, 1],
                           time_steady=40.0, peak_support=2, max_peaks=64)
    save = solver.save_times(torch.float64).numpy()
    wb = int(np.nonzero(save >= 40.0)[0][0])
    want = O.solve_batch(O.SYS_DUFFING, y0.numpy(), np.array([DUFFING.params]), save, (0.0, 60.0), 1e-10, 1e-10,
                         keep_full=True)
    assert od.peak_values.shape[1:] == (48, 2) and od.time_steady == 40.0
    for b in range(48):
        for d in range(2):
            ref = O.peak_values(want["y"][wb:, b, d], 2)
            assert int(od.peak_counts[b, d]) == len(ref)
            got = od.peak_values[: len(ref), b, d].cpu().numpy()
            np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7)
            assert torch.isnan(od.peak_values[len(ref):, b, d]).all()


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("feats", [[(0, L.FEAT_MAX, 0.0), (0, L.FEAT_STD, 0.0)],
                                   [(0, L.FEAT_MEAN, 0.0), (1, L.FEAT_LOG_DELTA, 0.0), (1, L.FEAT_LAST, 0.0)],
                                   [(0, L.FEAT_CROSSINGS, 0.0), (0, L.FEAT_MAX, 0.0)]],
                         ids=["one_state", "two_states", "crossings"])
def test_features_are_bit_identical_across_schedules(feats, precision):
    """Plain, queue and probed schedules write the same step records (explicit FMAs,
    same step sequence) and sampling reduces them the same way: the features are
    bit-identical whichever schedule ran.  With one or two feature states and no
    crossing counts the probed main phase samples finished trajectories itself
    (drained sampling); with crossings the sampling pass after it does."""
    case = DUFFING
    y0 = seeded_ics(case, 3000, 17).double().numpy()
    save = case.save_ts().numpy()
    t_span = (case.t_span[0], float(save[-1]))
    rtol = case.rtol if precision == L.PREC_FP64 else 1e-6
    kw = dict(precision=precision, win_begin=case.win_begin(), features=feats)
    ref = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, t_span, rtol, case.atol,
                    schedule=L.SCHED_PLAIN, **kw)
    for sched in (L.SCHED_QUEUE, L.SCHED_PROBED):
        got = gpu_solve(case.oracle_sys, y0, np.array([case.params]), save, t_span, rtol, case.atol,
                        schedule=sched, **kw)
        np.testing.assert_array_equal(got["features"], ref["features"])
        np.testing.assert_array_equal(got["status"], ref["status"])


@pytest.mark.parametrize("schedule,dense", [(L.SCHED_QUEUE, L.DENSE_DEFERRED), (L.SCHED_QUEUE, L.DENSE_INLINE),
                                            (L.SCHED_PROBED, L.DENSE_DEFERRED)])
@pytest.mark.parametrize("refill", [1, 8])
def test_lane_refill_is_bit_identical_to_whole_warp_refill(schedule, dense, refill):
    """Refilling idle lanes from the queue (a warp takes new positions once `refill`
    of its lanes are idle) changes which lane integrates which trajectory, never a
    trajectory's steps: statuses, step counts, features and final states equal those
    of the whole-warp schedule, with trajectories that stop early (unbounded runaways
    of the broken-butterfly Lorenz system, a NaN IC, a step budget) among them."""
    rng = np.random.default_rng(17)
    y0 = rng.uniform(-20.0, 20.0, (3000, 3))
    y0[5] = np.nan
    params = np.array([[0.12, 0.0, -0.6]])  # sigma, r, b: runaway trajectories
    save = np.linspace(0.0, 30.0, 301)
    feats = [(0, L.FEAT_MEAN, 0.0), (2, L.FEAT_MAX, 0.0), (1, L.FEAT_STD, 0.0)]
    kw = dict(precision=L.PREC_MIXED, schedule=schedule, dense_mode=dense, win_begin=100, features=feats,
              unbounded_thr=200.0, max_steps=3000)
    ref = gpu_solve(O.SYS_LORENZ, y0, params, save, (0.0, 30.0), 1e-6, 1e-6, **kw)
    got = gpu_solve(O.SYS_LORENZ, y0, params, save, (0.0, 30.0), 1e-6, 1e-6, refill_lanes=refill, **kw)
    assert len(set(ref["status"].tolist())) >= 2  # early stops are among them
    np.testing.assert_array_equal(got["status"], ref["status"])
    np.testing.assert_array_equal(got["steps"], ref["steps"])
    np.testing.assert_array_equal(got["features"], ref["features"])
    np.testing.assert_array_equal(got["y_final"], ref["y_final"])
