"""Pin the FP64 CPU oracle to the reference's golden vectors (CPU only)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.helpers import (
    DUFFING,
    PENDULUM,
    knn_labels,
    oracle_case_features,
    seeded_ics,
)

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_seeded_ics_reproduce_reference_fixture():
    """torch.manual_seed(42); torch.rand reproduces the fixture ICs (sampler.py:56-65)."""
    for case, name in ((PENDULUM, "labels_pendulum_case1.npz"), (DUFFING, "labels_duffing_main.npz")):
        g = np.load(GOLDEN / name)
        y0 = seeded_ics(case, 4000, seed=42)
        np.testing.assert_allclose(y0.numpy(), g["ics"], atol=1e-6)


def test_oracle_pendulum_labels_match_reference_exactly():
    """Pendulum case 1 (tests/integration/pendulum/test_pendulum.py:21-47): FP 602 / LC 3398."""
    g = np.load(GOLDEN / "labels_pendulum_case1.npz")
    y0 = seeded_ics(PENDULUM, 4000, seed=42).double().numpy()
    feats, tfeats, _ = oracle_case_features(PENDULUM, y0)
    pred = knn_labels(tfeats, feats)
    assert (pred == g["labels"]).all()
    np.testing.assert_array_equal(np.bincount(pred, minlength=2), g["counts"])


def test_oracle_duffing_labels_match_reference():
    """Duffing (tests/integration/duffing/test_duffing.py): MCC >= 0.95 and per-class counts
    within 2 of the reference's FP32 JAX labels (the oracle is FP64)."""
    from sklearn.metrics import matthews_corrcoef

    g = np.load(GOLDEN / "labels_duffing_main.npz")
    y0 = seeded_ics(DUFFING, 4000, seed=42).double().numpy()
    feats, tfeats, _ = oracle_case_features(DUFFING, y0)
    pred = knn_labels(tfeats, feats)
    assert matthews_corrcoef(g["labels"], pred) >= 0.99
    assert (pred != g["labels"]).sum() <= 8
    assert np.abs(np.bincount(pred, minlength=5) - g["counts"]).max() <= 2


def test_oracle_pendulum_n50_prefix():
    """N=50 at seed 42 on the CPU generator: the first 50 fixture labels (9 FP / 41 LC).

    The reference's test_n50 (tests/integration/pendulum/test_pendulum.py:109-124)
    quotes FP 0.12 +- 0.05 from a run whose sampler drew on its setup device; the
    CPU generator's first 50 ICs are the fixture's first 50 rows, which hold 9 FP."""
    g = np.load(GOLDEN / "labels_pendulum_case1.npz")
    y0 = seeded_ics(PENDULUM, 50, seed=42).double().numpy()
    feats, tfeats, _ = oracle_case_features(PENDULUM, y0)
    pred = knn_labels(tfeats, feats)
    assert (pred == g["labels"][:50]).all()
    assert np.bincount(pred, minlength=2).tolist() == [9, 41]


def test_oracle_exponential_decay_known_answers():
    """e^-1 and e^-2 at t=1 (tests/unit/solvers/test_solver.py:138,163,215-216)."""
    save = np.linspace(0.0, 1.0, 11)
    r = O.solve_batch(O.SYS_LINEAR, np.array([[1.0], [1.0]]), np.array([[-1.0], [-2.0]]), save, (0, 1), 1e-8, 1e-6,
                      param_index=np.array([0, 1]), keep_full=True)
    np.testing.assert_allclose(r["y"][-1, :, 0], [np.exp(-1), np.exp(-2)], rtol=0, atol=1e-6)
    np.testing.assert_allclose(r["y"][:, 0, 0], np.exp(-save), rtol=0, atol=1e-6)


def test_oracle_matches_reference_scipy_trajectories():
    """Short non-chaotic horizon vs the reference's ScipyParallelSolver (RK45, rtol 1e-11)."""
    g = np.load(GOLDEN / "scipy_reference.npz")
    for key, sys_id, p in (("pendulum", O.SYS_PENDULUM, [0.1, 0.5, 1.0]), ("duffing", O.SYS_DUFFING, [0.08, 1.0, 0.2])):
        y0 = g[f"{key}_y0"].astype(np.float64)
        t = g[f"{key}_t"]
        r = O.solve_batch(sys_id, y0, np.array([p]), t, (0.0, float(t[-1])), 1e-11, 1e-12, keep_full=True)
        np.testing.assert_allclose(r["y"], g[f"{key}_y"], rtol=2e-7, atol=2e-7)


@pytest.mark.parametrize(
    "name,kind,param",
    [
        ("median", 0, 0.0),
        ("mean", 1, 0.0),
        ("standard_deviation", 2, 0.0),
        ("variance", 3, 0.0),
        ("root_mean_square", 4, 0.0),
        ("maximum", 5, 0.0),
        ("absolute_maximum", 6, 0.0),
        ("minimum", 7, 0.0),
        ("delta", 8, 0.0),
        ("log_delta", 9, 0.0),
        ("amplitude", 10, 0.0),
        ("number_crossing_m_0", 11, 0.0),
        ("number_crossing_m_1", 11, 1.0),
        ("sum_values", 14, 0.0),
        ("abs_energy", 15, 0.0),
        ("length", 16, 0.0),
        ("variation_coefficient", 17, 0.0),
        ("quantile_0.1", 18, 0.1),
        ("quantile_0.75", 18, 0.75),
        ("kurtosis", 19, 0.0),
        ("skewness", 20, 0.0),
        ("absolute_sum_of_changes", 21, 0.0),
        ("mean_abs_change", 22, 0.0),
        ("mean_change", 23, 0.0),
        ("mean_second_derivative_central", 24, 0.0),
        ("count_above_mean", 25, 0.0),
        ("count_below_mean", 26, 0.0),
        ("count_above_0", 27, 0.0),
        ("count_below_0.5", 28, 0.5),
        ("number_peaks_1", 29, 1.0),
        ("number_peaks_3", 29, 3.0),
        ("autocorrelation_1", 30, 1.0),
        ("autocorrelation_7", 30, 7.0),
        ("ratio_beyond_r_sigma_1", 31, 1.0),
        *[(f"fft_coefficient_{a}_{k}", 32 + i, float(k))
          for i, a in enumerate(("real", "imag", "abs", "angle")) for k in (0, 1, 7, 128, 129)],
        *[(f"linear_trend_{a}", 36 + i, 0.0) for i, a in enumerate(("slope", "intercept", "rvalue", "pvalue", "stderr"))],
        ("first_location_of_maximum", 41, 0.0),
        ("first_location_of_minimum", 42, 0.0),
        ("last_location_of_maximum", 43, 0.0),
        ("last_location_of_minimum", 44, 0.0),
        ("cid_ce_true", 45, 1.0),
        ("cid_ce_false", 45, 0.0),
        ("c3_1", 46, 1.0),
        ("c3_5", 46, 5.0),
        ("c3_200", 46, 200.0),
        ("time_reversal_asymmetry_statistic_2", 47, 2.0),
        *[(f"spkt_welch_density_{k}", 48, float(k)) for k in (2, 5, 128, 129)],
        *[(f"large_standard_deviation_{r}", 49, r) for r in (0.1, 0.25, 0.3)],
        *[(f"symmetry_looking_{r}", 50, r) for r in (0.05, 0.5)],
        *[(f"index_mass_quantile_{q}", 51, q) for q in (0.1, 0.5, 0.9)],
        ("longest_strike_above_mean", 52, 0.0),
        ("longest_strike_below_mean", 53, 0.0),
        ("has_duplicate_max", 54, 0.0),
        ("has_duplicate_min", 55, 0.0),
        ("binned_entropy_10", 56, 10.0),
        ("binned_entropy_37", 56, 37.0),
        *[(f"mean_n_absolute_max_{k}", 57, float(k)) for k in (1, 3, 7)],
        ("benford_correlation", 58, 0.0),
    ],
)
def test_oracle_window_features_match_reference_calculators(name, kind, param):
    g = np.load(GOLDEN / "features_reference.npz")
    x = g["x"]
    want = g[name]
    got = np.array([[O.window_feature(kind, param, x[:, b, s]) for s in range(x.shape[2])] for b in range(x.shape[1])])
    # count_above / count_below / ratio_beyond_r_sigma: the reference averages a
    # boolean mask in FP32 (.float().mean()), divides the extreme locations as FP32
    # (idx.float() / n) and counts bins and digits in FP32 one-hot sums (binned
    # entropy, Benford): exact to FP32 rounding only.  The FFT coefficients
    # come from torch's FFT (another summation order): 1e-10 of the window's scale.
    fp32 = name.startswith(("count_above_", "count_below_", "ratio_beyond", "first_location", "last_location",
                            "index_mass_quantile", "binned_entropy", "benford"))
    tol = 2e-7 if fp32 else 1e-12
    atol = 1e-12
    if name.startswith("fft_coefficient_angle"):
        # the angle of a coefficient that vanishes (a constant window at k > 0) is
        # rounding noise in both: compared where the magnitude is resolved
        mag = g["fft_coefficient_abs_" + name.rsplit("_", 1)[1]]
        keep = mag > 1e-8 * np.abs(x).sum(axis=0)
        np.testing.assert_allclose(got[keep], want[keep], rtol=0.0, atol=1e-9)
        return
    if name.startswith(("fft_coefficient", "spkt_welch")):
        tol, atol = 1e-10, 1e-10 * np.abs(x).sum(axis=0).max()
    np.testing.assert_allclose(got, want, rtol=tol, atol=atol)


@pytest.mark.parametrize(
    "name, src, kind, param",
    [
        ("has_duplicate", "x", 59, 0.0),
        ("rep_has_duplicate", "x_rep", 59, 0.0),
        ("rep_percentage_of_reoccurring_datapoints_to_all_datapoints", "x_rep", 60, 0.0),
        ("rep_percentage_of_reoccurring_values_to_all_values", "x_rep", 61, 0.0),
        ("rep_sum_of_reoccurring_data_points", "x_rep", 62, 0.0),
        ("rep_sum_of_reoccurring_values", "x_rep", 63, 0.0),
        ("rep_ratio_value_number_to_time_series_length", "x_rep", 64, 0.0),
        ("ratio_value_number_to_time_series_length", "x", 64, 0.0),
        ("scaled_has_variance_larger_than_standard_deviation", "x_scaled", 65, 0.0),
        *[(f"rep_count_value_{v}", "x_rep", 66, v) for v in (0.0, 0.5, -1.0)],
    ],
)
def test_oracle_repeated_value_features_match_reference_calculators(name, src, kind, param):
    """Duplicates and reoccurring values on a window rounded to a 0.5 grid (one
    column holds a NaN, which equals nothing and turns both sums into NaN).  The
    reference returns its counts and ratios in FP32 (.float() masks), so those
    match to FP32 rounding; the sums run in the window's FP64."""
    g = np.load(GOLDEN / "features_reference.npz")
    x = g[src]
    want = g[name]
    got = np.array([[O.window_feature(kind, param, x[:, b, s]) for s in range(x.shape[2])] for b in range(x.shape[1])])
    assert np.array_equal(np.isnan(got), np.isnan(want))
    np.testing.assert_allclose(got, want, rtol=2e-7 if want.dtype == np.float32 else 1e-12, atol=1e-12)
    if src == "x_rep":
        assert np.isnan(want[2, 1]) == (kind in (62, 63))


_CQ_KIND = {(False, "mean"): 73, (False, "var"): 74, (True, "mean"): 75, (True, "var"): 76}


@pytest.mark.parametrize(
    "name, src, kind, param, param2",
    [
        *[(f"partial_autocorrelation_{k}", "x", 67, float(k), 0.0) for k in (0, 1, 2, 5, 9)],
        *[(f"agg_autocorrelation_{f}_{m}", "x", 68 + i, float(m), 0.0)
          for i, f in enumerate(("mean", "median", "var")) for m in (7, 40)],
        *[(f"energy_ratio_by_chunks_{k}_{i}", "x", 71, float(k), float(i))
          for (k, i) in ((10, 0), (10, 3), (10, 9), (3, 2), (300, 0))],
        *[(f"count_in_range_{lo}_{hi}", "x", 72, lo, hi) for (lo, hi) in ((-1.0, 1.0), (-1e12, 0.0), (0.0, 1e12))],
        ("rep_count_in_range_-1.0_1.0", "x_rep", 72, -1.0, 1.0),
        *[(f"change_quantiles_{ql}_{qh}_{b}_{f}", "x", _CQ_KIND[(b, f)], ql, qh)
          for (ql, qh) in ((0.0, 0.2), (0.2, 0.8), (0.4, 1.0)) for b in (False, True) for f in ("mean", "var")],
        *[(f"rep_change_quantiles_0.2_0.8_{b}_{f}", "x_rep", _CQ_KIND[(b, f)], 0.2, 0.8)
          for b in (False, True) for f in ("mean", "var")],
        *[(f"periodic_autocorrelation_periodicity_{o}_{m}_{t}", "x_periodic", 77 + i, float(m), t)
          for i, o in enumerate(("strength", "period")) for (m, t) in ((2, 0.3), (10, 0.5), (2, 0.9))],
        *[(f"autocorrelation_periodicity_{o}", "x", 77 + i, 2.0, 0.3) for i, o in enumerate(("strength", "period"))],
        *[(f"{tag}_{name}", src, kind, 0.0, 0.0)
          for tag, src in (("x", "x"), ("periodic", "x_periodic"), ("even", "x_even"))
          for name, kind in (("spectral_frequency_ratio", 79), ("fft_aggregated_centroid", 80),
                             ("fft_aggregated_variance", 81), ("fft_aggregated_skew", 82),
                             ("fft_aggregated_kurtosis", 83))],
        *[(f"{tag}_{name}", src, kind, p1, p2)
          for tag, src in (("x", "x"), ("periodic", "x_periodic"))
          for name, kind, p1, p2 in (("fourier_entropy", 84, 10.0, 0.0),
                                     *[(f"permutation_entropy_{t}_{d}", 85, float(t), float(d))
                                       for (t, d) in ((1, 3), (1, 4), (2, 5), (1, 7), (3, 3))],
                                     *[(f"lempel_ziv_complexity_{b}", 86, float(b), 0.0) for b in (2, 3, 5, 10, 100)])],
        *[(f"{tag}_agg_linear_trend_{a}_{c}_{f}", src, 87 + fi, float(c), float(ai))
          for tag, src in (("x", "x"), ("periodic", "x_periodic"))
          for ai, a in enumerate(("slope", "intercept", "rvalue", "pvalue", "stderr")) for c in (5, 50, 200)
          for fi, f in enumerate(("mean", "var", "min", "max"))],
        *[(f"x_linear_trend_timewise_{a}", "x", 36 + i, 0.0, 0.0) for i, a in ((0, "slope"), (2, "rvalue"))],
        *[(f"{tag}_cwt_coefficients_{w}_{c}", src, 92, float(w), float(c))
          for tag, src in (("x", "x"), ("periodic", "x_periodic")) for w in (2, 5, 10, 20) for c in (0, 3, 14, 128, 256)],
        ("x_cwt_coefficients_missing_width", "x", 92, 2.0, -1.0),
        *[(f"{tag}_friedrich_coefficients_{m}_{c}", src, 93, float(m), float(c))
          for tag, src in (("x", "x"), ("periodic", "x_periodic")) for m in (1, 3) for c in range(m + 2)],
        *[(f"{tag}_max_langevin_fixed_point_{m}", src, 94, float(m), 0.0)
          for tag, src in (("x", "x"), ("periodic", "x_periodic")) for m in (1, 3)],
        *[(f"{tag}_augmented_dickey_fuller_{a}", src, 95 + i, 0.0, 0.0)
          for tag, src in (("x", "x"), ("periodic", "x_periodic")) for i, a in enumerate(("teststat", "pvalue", "usedlag"))],
        *[(f"{tag}_number_cwt_peaks_{w}", src, 98, float(w), 0.0)
          for tag, src in (("x", "x"), ("periodic", "x_periodic"), ("rep", "x_rep")) for w in (1, 5, 200)],
        *[(f"{tag}_ar_coefficient_{k}_{c}", src, 91, float(k), float(c))
          for tag, src in (("x", "x"), ("periodic", "x_periodic"))
          for (k, c) in ((10, 0), (10, 3), (10, 9), (10, 10), (1, 0), (4, 2))],
    ],
)
def test_oracle_two_parameter_and_acf_features_match_reference_calculators(name, src, kind, param, param2):
    """Partial and aggregated autocorrelation, autocorrelation periodicity (noisy
    sine waves of 16 periods, one constant column), spectral frequency ratio and
    aggregated spectrum moments (odd and even lengths), Fourier and permutation
    entropy, Lempel-Ziv complexity (exact phrase counts), trends of chunk
    aggregates, AR coefficients (Yule-Walker), Ricker-wavelet coefficients (the
    reference's FP32 prefactor), Friedrich coefficients and the Langevin fixed
    point, augmented Dickey-Fuller, CWT-peak counts (ties and a NaN on the 0.5
    grid), energy ratio of a chunk,
    count in a range and change quantiles.  The reference's autocorrelations come from a
    zero-padded FFT (another summation order than the oracle's direct lag sums):
    1e-10 absolute on values bounded by 1; count_in_range counts in FP32; the
    rest 1e-12 relative.  On the 0.5-grid copy the corridor bounds of change
    quantiles are sample values, so ties at both bounds are inside."""
    g = np.load(GOLDEN / "features_reference.npz")
    x = g[src]
    want = g[name]
    got = np.array([[O.window_feature(kind, param, x[:, b, s], param2) for s in range(x.shape[2])]
                    for b in range(x.shape[1])])
    if 67 <= kind <= 70 or kind == 77:
        np.testing.assert_allclose(got, want, rtol=0.0, atol=1e-10)
    elif kind in (91, 93):  # linear systems solved by torch's LU against the oracle's elimination
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)
    elif 80 <= kind <= 84:  # torch's FFT against the oracle's direct sums
        np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12)
    else:
        np.testing.assert_allclose(got, want, rtol=2e-7 if want.dtype == np.float32 else 1e-12, atol=1e-12)


@pytest.mark.parametrize("src", ["x", "x_periodic"])
@pytest.mark.parametrize("emb, lag, n_rvals", [(4, 1, 50), (2, 3, 20), (6, 2, 50)])
def test_oracle_correlation_dimension_matches_reference(src, emb, lag, n_rvals):
    """Grassberger-Procaccia correlation dimension (ts_torch/torch_corr_dim.py).  The
    reference fits the slope in FP32: 1e-4 relative, and where the exact slope is 0
    (every radius holding the same pair count) its cancellation leaves up to 2e-3.
    A constant window makes the fit degenerate; the reference then returns 0 or
    NaN depending on its FP32 rounding, the oracle NaN, so those columns are skipped."""
    g = np.load(GOLDEN / "features_reference.npz")
    x = g[src]
    tag = "x" if src == "x" else "periodic"
    want = g[f"{tag}_correlation_dimension_{emb}_{lag}_{n_rvals}"].astype(np.float64)
    got = np.array([[O.window_feature(99, float(emb), x[:, b, s], float(lag * 1024 + n_rvals)) for s in range(2)]
                    for b in range(x.shape[1])])
    live = x.std(axis=0) > 0
    assert live.sum() >= 30
    np.testing.assert_allclose(got[live], want[live], rtol=1e-4, atol=2e-3)
    assert np.isnan(got[~live]).all()


@pytest.mark.parametrize("src", ["x", "x_periodic"])
@pytest.mark.parametrize("emb, lag, tlen", [(10, 1, 20), (4, 2, 10), (3, 1, 40)])
def test_oracle_lyapunov_r_matches_reference(src, emb, lag, tlen):
    """Largest Lyapunov exponent by Rosenstein's method (ts_torch/torch_lyapunov_r.py):
    the reference keeps the divergence curve and its fit in FP32, so 1e-4 relative
    (the differences seen are below 6e-6)."""
    g = np.load(GOLDEN / "features_reference.npz")
    x = g[src]
    tag = "x" if src == "x" else "periodic"
    want = g[f"{tag}_lyapunov_r_{emb}_{lag}_{tlen}"].astype(np.float64)
    got = np.array([[O.window_feature(100, float(emb * 1024 + tlen), x[:, b, s], float(lag)) for s in range(2)]
                    for b in range(x.shape[1])])
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-6)


def test_oracle_quantile_even_length():
    g = np.load(GOLDEN / "features_reference.npz")
    x = g["x_even"]
    got = np.array([[O.window_feature(18, 0.3, x[:, b, s]) for s in range(2)] for b in range(x.shape[1])])
    np.testing.assert_allclose(got, g["quantile_even_0.3"], rtol=1e-12, atol=1e-12)


def test_oracle_median_even_length_is_lower_median():
    g = np.load(GOLDEN / "features_reference.npz")
    x = g["x_even"]
    got = np.array([[O.window_feature(0, 0.0, x[:, b, s]) for s in range(2)] for b in range(x.shape[1])])
    np.testing.assert_array_equal(got, g["median_even"])


def test_oracle_status_codes():
    save = np.linspace(0.0, 10.0, 5)
    # max_steps
    r = O.solve_batch(O.SYS_PENDULUM, np.array([[0.1, 0.0]]), np.array([[0.1, 0.5, 1.0]]), save, (0, 10), 1e-8, 1e-6,
                      max_steps=10)
    assert r["status"][0] == O.STATUS_MAX_STEPS
    # non-finite initial condition
    r = O.solve_batch(O.SYS_PENDULUM, np.array([[np.nan, 0.0]]), np.array([[0.1, 0.5, 1.0]]), save, (0, 10), 1e-8, 1e-6)
    assert r["status"][0] == O.STATUS_NONFINITE
    # unbounded event on exponential growth
    r = O.solve_batch(O.SYS_LINEAR, np.array([[1.0]]), np.array([[5.0]]), save, (0, 10), 1e-8, 1e-6, unbounded_thr=1e6,
                      keep_full=True)
    assert r["status"][0] == O.STATUS_UNBOUNDED
    assert np.isinf(r["y"][-1, 0, 0])


def test_oracle_cross_layout_equals_explicit_expansion():
    """IC-major expansion (src/pybasin/solvers/base.py:155-159)."""
    y0 = np.array([[0.5, 0.0], [2.0, 1.0]])
    P = np.array([[0.1, 0.3, 1.0], [0.1, 0.7, 1.0], [0.2, 0.5, 1.0]])
    save = np.linspace(0.0, 5.0, 6)
    idx = np.tile(np.arange(3), 2)
    r = O.solve_batch(O.SYS_PENDULUM, np.repeat(y0, 3, axis=0), P, save, (0, 5), 1e-9, 1e-9, param_index=idx,
                      keep_full=True)
    for ic in range(2):
        for p in range(3):
            one = O.solve_batch(O.SYS_PENDULUM, y0[ic : ic + 1], P[p : p + 1], save, (0, 5), 1e-9, 1e-9, keep_full=True)
            np.testing.assert_array_equal(r["y"][:, ic * 3 + p], one["y"][:, 0])


def test_torch_linspace_save_times_are_float32_rounded():
    """The reference's save grid is linspace in y0's dtype (base.py:113-127)."""
    s32 = torch.linspace(900, 1000, 5000, dtype=torch.float32).double()
    s64 = torch.linspace(900, 1000, 5000, dtype=torch.float64)
    assert (s32 - s64).abs().max() > 1e-6


def test_friction_labels_equal_reference_fixture():
    """Friction case 1 (tests/integration/friction/test_friction.py, seed 42, N = 4000):
    max |v| over t in [400, 500] > 0.2 -> LC (friction_feature_extractor.py:17-41)."""
    d = np.load(GOLDEN / "labels_friction_case1.npz")
    save = torch.linspace(400, 500, 500, dtype=torch.float32).double().numpy()
    p = np.array([[1.5, 0.05, 2.0, 0.5, 0.0, 0.5]])  # setup_friction_system.py:19-26
    r = O.solve_batch(O.SYS_FRICTION, d["ics"].astype(np.float64), p, save, (0.0, 500.0), 1e-8, 1e-6,
                      features=[(1, 6, 0.0)])
    labels = (r["features"][:, 0] > 0.2).astype(np.int8)
    assert (r["status"] == 0).all()
    np.testing.assert_array_equal(labels, d["labels"])
    assert np.bincount(labels).tolist() == d["counts"].tolist() == [1266, 2734]
