"""Generate the golden fixtures under tests/golden/ from the pybasin reference.

Run once in a container where the reference tree is present:

    python tests/golden/make_golden.py /root/reference

(the reference tree is a required argument, or the PYBASIN_REFERENCE
environment variable).
It imports the reference (with empty stand-in modules for the two imports that
are not installed, ``torchdiffeq`` and ``matplotlib``; neither is on the paths
used here) and writes:

* ``labels_pendulum_case1.npz`` / ``labels_duffing_main.npz`` /
  ``labels_friction_case1.npz`` — the reference's seeded label fixtures
  (tests/integration/pendulum/ground_truths/case1/main_pendulum_case1.csv,
  tests/integration/duffing/ground_truths/main/main_duffing.csv,
  tests/integration/friction/ground_truths/main/main_friction.csv; seed 42,
  N=4000) as class indices plus class names, with the basin-stability counts of
  main_pendulum_case1.json / main_duffing_supervised.json / main_friction_case1.json.
* ``features_reference.npz`` — outputs of the reference's own feature
  calculators (src/pybasin/ts_torch/calculators/*.py) on seeded random windows
  (and a copy rounded to a 0.5 grid, so that values repeat), to pin the statistics.
* ``rossler_network_reference.npz`` — the reference's 100-node / 400-edge graph
  (case_studies/rossler_network/rossler_network_topology.py) and the paper's
  basin-stability values per coupling K it tests against
  (case_studies/rossler_network/setup_rossler_network_system.py).
* ``scipy_reference.npz`` — the reference's ScipyParallelSolver
  (src/pybasin/solvers/scipy_solver.py) on a few seeded pendulum and Duffing ICs
  over a short horizon at tight tolerance, to pin trajectories.
"""

from __future__ import annotations

import json
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np
import pandas as pd
import torch

OUT = Path(__file__).resolve().parent


def _install_stubs() -> None:
    tmp = Path(tempfile.mkdtemp(prefix="pb_stubs_"))
    (tmp / "torchdiffeq").mkdir()
    (tmp / "torchdiffeq" / "__init__.py").write_text(
        "def odeint(*a, **k):\n    raise RuntimeError('torchdiffeq is not installed')\n"
    )
    mpl = tmp / "matplotlib"
    mpl.mkdir()
    (mpl / "__init__.py").write_text("def use(*a, **k):\n    pass\n")
    (mpl / "pyplot.py").write_text("def __getattr__(name):\n    raise AttributeError(name)\n")
    (mpl / "figure.py").write_text("class Figure: pass\n")
    (mpl / "axes.py").write_text("class Axes: pass\n")
    (mpl / "colors.py").write_text("def __getattr__(name):\n    raise AttributeError(name)\n")
    sys.path.insert(0, str(tmp))


def _labels(ref: Path, csv: str, js: str, classes: list[str], name: str) -> None:
    df = pd.read_csv(ref / csv)
    meta = json.loads((ref / js).read_text())
    label_map = meta.get("label_map", {})
    idx = {c: i for i, c in enumerate(classes)}
    lab = np.array([idx[s] for s in df["label"].astype(str)], dtype=np.int8)
    counts = {label_map.get(d["label"], d["label"]): int(d["absNumMembers"]) for d in meta["data"]}
    np.savez_compressed(
        OUT / name,
        labels=lab,
        classes=np.array(classes),
        ics=df[["x1", "x2"]].to_numpy(np.float32),
        counts=np.array([counts.get(c, 0) for c in classes], dtype=np.int64),
    )


def _features(ref: Path) -> None:
    from pybasin.ts_torch.calculators import torch_features_autocorrelation as ac
    from pybasin.ts_torch.calculators import torch_features_change as ch
    from pybasin.ts_torch.calculators import torch_features_count as cn
    from pybasin.ts_torch.calculators import torch_features_pattern as pat
    from pybasin.ts_torch.calculators import torch_features_statistical as st
    from pybasin.ts_torch.calculators import torch_features_advanced as ad
    from pybasin.ts_torch.calculators import torch_features_boolean as bo
    from pybasin.ts_torch.calculators import torch_features_dynamical as dy
    from pybasin.ts_torch.calculators import torch_features_entropy_complexity as ec
    from pybasin.ts_torch.calculators import torch_features_frequency as fq
    from pybasin.ts_torch.calculators import torch_features_location as lo
    from pybasin.ts_torch.calculators import torch_features_reocurrance as re
    from pybasin.ts_torch.calculators import torch_features_trend as tr

    g = torch.Generator().manual_seed(1234)
    n_t, n_b = 257, 16
    x = torch.randn(n_t, n_b, 2, generator=g, dtype=torch.float64) * 3.0 + 0.5
    x[:, 3, 0] = 2.0  # constant row
    x[::2, 5, 1] = -x[::2, 5, 1]  # sign flips for crossings
    even = torch.randn(256, n_b, 2, generator=g, dtype=torch.float64)  # even length: lower median
    # a window on a 0.5 grid, so values repeat (duplicate and reoccurrence features),
    # with one NaN sample; and a scaled copy whose standard deviations straddle 1
    rep = torch.round(x * 2.0) / 2.0
    rep[7, 2, 1] = float("nan")
    scaled = x * 0.35
    # noisy sine waves of 16 periods (6.5 to 36.5 samples), for the periodicity features
    tt = torch.arange(n_t, dtype=torch.float64)
    per = torch.sin(2.0 * torch.pi * tt[:, None, None] / (6.5 + 2.0 * torch.arange(n_b, dtype=torch.float64))[None, :, None]
                    + torch.tensor([0.0, 1.0], dtype=torch.float64)) + 0.3 * torch.randn(n_t, n_b, 2, generator=g,
                                                                                          dtype=torch.float64)
    per[:, 4, 1] = 0.25  # constant: no peak
    res = {
        "x": x.numpy(),
        "x_even": even.numpy(),
        "median": st.median(x).numpy(),
        "median_even": st.median(even).numpy(),
        "mean": st.mean(x).numpy(),
        "standard_deviation": st.standard_deviation(x).numpy(),
        "variance": st.variance(x).numpy(),
        "root_mean_square": st.root_mean_square(x).numpy(),
        "maximum": st.maximum(x).numpy(),
        "absolute_maximum": st.absolute_maximum(x).numpy(),
        "minimum": st.minimum(x).numpy(),
        "delta": st.delta(x).numpy(),
        "log_delta": st.log_delta(x).numpy(),
        "amplitude": st.amplitude(x).numpy(),
        "number_crossing_m_0": pat.number_crossing_m(x, 0).numpy(),
        "number_crossing_m_1": pat.number_crossing_m(x, 1).numpy(),
        # wider set (window features)
        "sum_values": st.sum_values(x).numpy(),
        "abs_energy": st.abs_energy(x).numpy(),
        "length": st.length(x).numpy(),
        "variation_coefficient": st.variation_coefficient(x).numpy(),
        "quantile_0.1": st.quantile(x, 0.1).numpy(),
        "quantile_0.75": st.quantile(x, 0.75).numpy(),
        "quantile_even_0.3": st.quantile(even, 0.3).numpy(),
        "kurtosis": st.kurtosis(x).numpy(),
        "skewness": st.skewness(x).numpy(),
        "absolute_sum_of_changes": ch.absolute_sum_of_changes(x).numpy(),
        "mean_abs_change": ch.mean_abs_change(x).numpy(),
        "mean_change": ch.mean_change(x).numpy(),
        "mean_second_derivative_central": ch.mean_second_derivative_central(x).numpy(),
        "count_above_mean": cn.count_above_mean(x).numpy(),
        "count_below_mean": cn.count_below_mean(x).numpy(),
        "count_above_0": cn.count_above(x, 0).numpy(),
        "count_below_0.5": cn.count_below(x, 0.5).numpy(),
        "number_peaks_1": pat.number_peaks(x, 1).numpy(),
        "number_peaks_3": pat.number_peaks(x, 3).numpy(),
        "autocorrelation_1": ac.autocorrelation(x, 1).numpy(),
        "autocorrelation_7": ac.autocorrelation(x, 7).numpy(),
        "ratio_beyond_r_sigma_1": st.ratio_beyond_r_sigma(x, 1.0).numpy(),
        # FFT coefficients, linear trend, extreme locations, cid_ce, c3, time reversal
        **{f"fft_coefficient_{a}_{k}": fq.fft_coefficient(x, k, a).numpy()
           for a in ("real", "imag", "abs", "angle") for k in (0, 1, 7, 128, 129)},
        **{f"linear_trend_{a}": tr.linear_trend(x, a).numpy()
           for a in ("slope", "intercept", "rvalue", "pvalue", "stderr")},
        "first_location_of_maximum": lo.first_location_of_maximum(x).numpy(),
        "first_location_of_minimum": lo.first_location_of_minimum(x).numpy(),
        "last_location_of_maximum": lo.last_location_of_maximum(x).numpy(),
        "last_location_of_minimum": lo.last_location_of_minimum(x).numpy(),
        "cid_ce_true": ec.cid_ce(x, True).numpy(),
        "cid_ce_false": ec.cid_ce(x, False).numpy(),
        "c3_1": ad.c3(x, 1).numpy(),
        "c3_5": ad.c3(x, 5).numpy(),
        "c3_200": ad.c3(x, 200).numpy(),
        "time_reversal_asymmetry_statistic_2": ad.time_reversal_asymmetry_statistic(x, 2).numpy(),
        **{f"spkt_welch_density_{k}": fq.spkt_welch_density(x, k).numpy() for k in (2, 5, 128, 129)},
        **{f"large_standard_deviation_{r}": bo.has_large_standard_deviation(x, r).numpy() for r in (0.1, 0.25, 0.3)},
        **{f"symmetry_looking_{r}": st.symmetry_looking(x, r).numpy() for r in (0.05, 0.5)},
        **{f"index_mass_quantile_{q}": lo.index_mass_quantile(x, q).numpy() for q in (0.1, 0.5, 0.9)},
        "longest_strike_above_mean": pat.longest_strike_above_mean(x).numpy(),
        "longest_strike_below_mean": pat.longest_strike_below_mean(x).numpy(),
        "has_duplicate_max": bo.has_duplicate_max(x).numpy(),
        "has_duplicate_min": bo.has_duplicate_min(x).numpy(),
        **{f"binned_entropy_{b}": ec.binned_entropy(x, b).numpy() for b in (10, 37)},
        **{f"mean_n_absolute_max_{k}": st.mean_n_absolute_max(x, k).numpy() for k in (1, 3, 7)},
        "benford_correlation": ad.benford_correlation(x).numpy(),
        # repeated values (torch_features_boolean.py, torch_features_reocurrance.py,
        # torch_features_count.py)
        "x_rep": rep.numpy(),
        "x_scaled": scaled.numpy(),
        "has_duplicate": bo.has_duplicate(x).numpy(),
        "rep_has_duplicate": bo.has_duplicate(rep).numpy(),
        "rep_percentage_of_reoccurring_datapoints_to_all_datapoints":
            re.percentage_of_reoccurring_datapoints_to_all_datapoints(rep).numpy(),
        "rep_percentage_of_reoccurring_values_to_all_values":
            re.percentage_of_reoccurring_values_to_all_values(rep).numpy(),
        "rep_sum_of_reoccurring_data_points": re.sum_of_reoccurring_data_points(rep).numpy(),
        "rep_sum_of_reoccurring_values": re.sum_of_reoccurring_values(rep).numpy(),
        "rep_ratio_value_number_to_time_series_length": re.ratio_value_number_to_time_series_length(rep).numpy(),
        "ratio_value_number_to_time_series_length": re.ratio_value_number_to_time_series_length(x).numpy(),
        **{f"rep_count_value_{v}": cn.count_value(rep, v).numpy() for v in (0.0, 0.5, -1.0)},
        "scaled_has_variance_larger_than_standard_deviation":
            bo.has_variance_larger_than_standard_deviation(scaled).numpy(),
        # autocorrelation family and the two-parameter features
        **{f"partial_autocorrelation_{k}": ac.partial_autocorrelation(x, k).numpy() for k in (0, 1, 2, 5, 9)},
        **{f"agg_autocorrelation_{f}_{m}": ac.agg_autocorrelation(x, m, f).numpy()
           for f in ("mean", "median", "var") for m in (7, 40)},
        **{f"energy_ratio_by_chunks_{k}_{i}": ad.energy_ratio_by_chunks(x, k, i).numpy()
           for (k, i) in ((10, 0), (10, 3), (10, 9), (3, 2), (300, 0))},
        **{f"count_in_range_{lo}_{hi}": cn.count_in_range(x, lo, hi).numpy()
           for (lo, hi) in ((-1.0, 1.0), (-1e12, 0.0), (0.0, 1e12))},
        "rep_count_in_range_-1.0_1.0": cn.count_in_range(rep, -1.0, 1.0).numpy(),
        **{f"change_quantiles_{ql}_{qh}_{b}_{f}": ch.change_quantiles(x, ql, qh, b, f).numpy()
           for (ql, qh) in ((0.0, 0.2), (0.2, 0.8), (0.4, 1.0)) for b in (False, True) for f in ("mean", "var")},
        **{f"rep_change_quantiles_0.2_0.8_{b}_{f}": ch.change_quantiles(rep, 0.2, 0.8, b, f).numpy()
           for b in (False, True) for f in ("mean", "var")},
        "x_periodic": per.numpy(),
        **{f"periodic_autocorrelation_periodicity_{o}_{m}_{t}":
           ac.autocorrelation_periodicity(per, m, t, o).numpy()
           for o in ("strength", "period") for (m, t) in ((2, 0.3), (10, 0.5), (2, 0.9))},
        **{f"autocorrelation_periodicity_{o}": ac.autocorrelation_periodicity(x, output=o).numpy()
           for o in ("strength", "period")},
        # spectra (odd and even lengths)
        **{f"{src}_spectral_frequency_ratio": fq.spectral_frequency_ratio(v).numpy()
           for src, v in (("x", x), ("periodic", per), ("even", even))},
        **{f"{src}_fft_aggregated_{a}": fq.fft_aggregated(v, a).numpy()
           for src, v in (("x", x), ("periodic", per), ("even", even))
           for a in ("centroid", "variance", "skew", "kurtosis")},
        # entropies and complexity
        **{f"{src}_fourier_entropy": ec.fourier_entropy(v, 10).numpy() for src, v in (("x", x), ("periodic", per))},
        **{f"{src}_permutation_entropy_{t}_{d}": ec.permutation_entropy(v, t, d).numpy()
           for src, v in (("x", x), ("periodic", per)) for (t, d) in ((1, 3), (1, 4), (2, 5), (1, 7), (3, 3))},
        **{f"{src}_lempel_ziv_complexity_{b}": ec.lempel_ziv_complexity(v, b).numpy()
           for src, v in (("x", x), ("periodic", per)) for b in (2, 3, 5, 10, 100)},
        # trends of chunk aggregates, AR coefficients
        **{f"{src}_agg_linear_trend_{a}_{c}_{f}": tr.agg_linear_trend(v, c, f, a).numpy()
           for src, v in (("x", x), ("periodic", per))
           for a in ("slope", "intercept", "rvalue", "pvalue", "stderr") for c in (5, 50, 200) for f in
           ("mean", "var", "min", "max")},
        **{f"{src}_linear_trend_timewise_{a}": tr.linear_trend_timewise(v, a).numpy()
           for src, v in (("x", x),) for a in ("slope", "rvalue")},
        **{f"{src}_cwt_coefficients_{w}_{c}": fq.cwt_coefficients(v, (w,), c, w).numpy()
           for src, v in (("x", x), ("periodic", per)) for w in (2, 5, 10, 20) for c in (0, 3, 14, 128, 256)},
        "x_cwt_coefficients_missing_width": fq.cwt_coefficients(x, (5,), 3, 2).numpy(),
        **{f"{src}_friedrich_coefficients_{m}_{c}": dy.friedrich_coefficients(v, m, 30.0, c).numpy()
           for src, v in (("x", x), ("periodic", per)) for m in (1, 3) for c in range(m + 2)},
        **{f"{src}_max_langevin_fixed_point_{m}": dy.max_langevin_fixed_point(v, m=m, r=30.0).numpy()
           for src, v in (("x", x), ("periodic", per)) for m in (1, 3)},
        **{f"{src}_augmented_dickey_fuller_{a}": tr.augmented_dickey_fuller(v, a).numpy()
           for src, v in (("x", x), ("periodic", per)) for a in ("teststat", "pvalue", "usedlag")},
        **{f"{src}_number_cwt_peaks_{w}": pat.number_cwt_peaks(v, w).numpy()
           for src, v in (("x", x), ("periodic", per), ("rep", rep)) for w in (1, 5, 200)},
        **{f"{src}_correlation_dimension_{e}_{l}_{r}": dy.correlation_dimension(v, e, l, r).numpy()
           for src, v in (("x", x), ("periodic", per)) for (e, l, r) in ((4, 1, 50), (2, 3, 20), (6, 2, 50))},
        **{f"{src}_lyapunov_r_{e}_{l}_{t}": dy.lyapunov_r(v, e, l, t, 1.0).numpy()
           for src, v in (("x", x), ("periodic", per)) for (e, l, t) in ((10, 1, 20), (4, 2, 10), (3, 1, 40))},
        **{f"{src}_ar_coefficient_{k}_{c}": tr.ar_coefficient(v, k, c).numpy()
           for src, v in (("x", x), ("periodic", per)) for (k, c) in ((10, 0), (10, 3), (10, 9), (10, 10), (1, 0),
                                                                       (4, 2))},
    }
    np.savez_compressed(OUT / "features_reference.npz", **res)


def _scipy(ref: Path) -> None:
    sys.path.insert(0, str(ref))
    from case_studies.duffing_oscillator.duffing_ode import DuffingODE  # noqa: F401  (torch variant)
    from case_studies.pendulum.pendulum_ode import PendulumNumpyODE
    from pybasin.solvers import ScipyParallelSolver
    from pybasin.solvers.numpy_ode_system import NumpyODESystem

    class DuffingNumpyODE(NumpyODESystem):  # the reference ships only torch/JAX Duffing variants
        def ode(self, t, y, p):
            return np.array([y[1], -p[0] * y[1] - p[1] * y[0] ** 3 + p[2] * np.cos(t)])

    out = {}
    torch.manual_seed(7)
    for key, ode, lo, hi in (
        ("pendulum", PendulumNumpyODE({"alpha": 0.1, "T": 0.5, "K": 1.0}), [-2.6, -10.0], [3.7, 10.0]),
        ("duffing", DuffingNumpyODE({"delta": 0.08, "k3": 1.0, "A": 0.2}), [-1.0, -0.5], [1.0, 1.0]),
    ):
        lo_t, hi_t = torch.tensor(lo), torch.tensor(hi)
        y0 = torch.rand(8, 2) * (hi_t - lo_t) + lo_t
        solver = ScipyParallelSolver(
            t_span=(0, 20), t_steps=41, n_jobs=1, rtol=1e-11, atol=1e-12, max_step=0.05, cache_dir=None
        )
        t, y = solver.integrate(ode, y0.double())
        out[f"{key}_y0"] = y0.numpy()
        out[f"{key}_t"] = t.double().numpy()
        out[f"{key}_y"] = y.double().numpy()
    np.savez_compressed(OUT / "scipy_reference.npz", **out)


def _rossler(ref: Path) -> None:
    """The reference's 100-node / 400-edge Rössler graph and the paper's S_B values,
    read as literals from the case-study sources (their modules import JAX)."""
    import ast

    def literal(path: Path, name: str):
        tree = ast.parse(path.read_text())
        for node in ast.walk(tree):
            if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == name for t in node.targets):
                v = node.value
                if isinstance(v, ast.Call):  # np.array([...])
                    v = v.args[0]
                return ast.literal_eval(v)
        raise KeyError(name)

    cs = ref / "case_studies" / "rossler_network"
    edges_str = literal(cs / "rossler_network_topology.py", "EDGE_LIST_STR")
    edges = np.array([[int(a), int(b)] for a, b in (e.split("-") for e in edges_str.split(", "))], dtype=np.int32)
    k_vals = np.array(literal(cs / "setup_rossler_network_system.py", "K_VALUES_FROM_PAPER"), dtype=np.float64)
    sb = np.array(literal(cs / "setup_rossler_network_system.py", "EXPECTED_SB_FROM_PAPER"), dtype=np.float64)
    np.savez_compressed(OUT / "rossler_network_reference.npz", edges=edges, k_values=k_vals, expected_sb=sb,
                        n_reference=np.int64(500))


def main() -> None:
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYBASIN_REFERENCE")
    if not src:
        sys.exit("usage: make_golden.py <reference tree> (or set PYBASIN_REFERENCE)")
    ref = Path(src)
    _install_stubs()
    sys.path.insert(0, str(ref / "src"))
    it = ref / "tests" / "integration"
    _labels(
        it,
        "pendulum/ground_truths/case1/main_pendulum_case1.csv",
        "pendulum/main_pendulum_case1.json",
        ["FP", "LC"],
        "labels_pendulum_case1.npz",
    )
    _labels(
        it,
        "duffing/ground_truths/main/main_duffing.csv",
        "duffing/main_duffing_supervised.json",
        [f"$\\bar{{y}}_{i}$" for i in range(1, 6)],
        "labels_duffing_main.npz",
    )
    _labels(
        it,
        "friction/ground_truths/main/main_friction.csv",
        "friction/main_friction_case1.json",
        ["FP", "LC"],
        "labels_friction_case1.npz",
    )
    _features(ref)
    _scipy(ref)
    _rossler(ref)
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
