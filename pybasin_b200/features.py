"""Fused steady-state features: configuration and the extractor side channel.

``FusedFeatureExtractor`` takes the constructor arguments of the reference's
``TorchFeatureExtractor`` (src/pybasin/ts_torch/torch_feature_extractor.py:86-127)
and produces the same columns, names (``state_{i}__{feature}``,
src/pybasin/feature_extractors/utils.py:34-73), imputation
(src/pybasin/ts_torch/torch_feature_utilities.py:60-94) and optional z-score
(torch_feature_extractor.py:269-285).  The statistics themselves are computed
inside the integration kernel; the solver attaches them to the ``y`` tensor it
returns and ``extract_features`` reads them back.
"""

from __future__ import annotations

import threading
from typing import Any

import torch

from pybasin_b200 import _lib as L
from pybasin_b200.engine import FeatureColumn

#: Feature names of src/pybasin/ts_torch/settings.py mapped to fused kernels.
FEATURE_KINDS: dict[str, int] = {
    "median": L.FEAT_MEDIAN,
    "mean": L.FEAT_MEAN,
    "standard_deviation": L.FEAT_STD,
    "variance": L.FEAT_VAR,
    "root_mean_square": L.FEAT_RMS,
    "maximum": L.FEAT_MAX,
    "absolute_maximum": L.FEAT_ABSMAX,
    "minimum": L.FEAT_MIN,
    "delta": L.FEAT_DELTA,
    "log_delta": L.FEAT_LOG_DELTA,
    "amplitude": L.FEAT_AMPLITUDE,
    "number_crossing_m": L.FEAT_CROSSINGS,
    "sum_values": L.FEAT_SUM,
    "abs_energy": L.FEAT_ABS_ENERGY,
    "length": L.FEAT_LENGTH,
    "variation_coefficient": L.FEAT_VARIATION_COEFF,
    "quantile": L.FEAT_QUANTILE,
    "kurtosis": L.FEAT_KURTOSIS,
    "skewness": L.FEAT_SKEWNESS,
    "absolute_sum_of_changes": L.FEAT_ABS_SUM_CHANGES,
    "mean_abs_change": L.FEAT_MEAN_ABS_CHANGE,
    "mean_change": L.FEAT_MEAN_CHANGE,
    "mean_second_derivative_central": L.FEAT_MEAN_SECOND_DERIV,
    "count_above_mean": L.FEAT_COUNT_ABOVE_MEAN,
    "count_below_mean": L.FEAT_COUNT_BELOW_MEAN,
    "count_above": L.FEAT_COUNT_ABOVE,
    "count_below": L.FEAT_COUNT_BELOW,
    "number_peaks": L.FEAT_NUMBER_PEAKS,
    "autocorrelation": L.FEAT_AUTOCORRELATION,
    "ratio_beyond_r_sigma": L.FEAT_RATIO_BEYOND_R_SIGMA,
    "first_location_of_maximum": L.FEAT_FIRST_LOC_MAX,
    "first_location_of_minimum": L.FEAT_FIRST_LOC_MIN,
    "last_location_of_maximum": L.FEAT_LAST_LOC_MAX,
    "last_location_of_minimum": L.FEAT_LAST_LOC_MIN,
    "cid_ce": L.FEAT_CID_CE,
    "c3": L.FEAT_C3,
    "time_reversal_asymmetry_statistic": L.FEAT_TIME_REVERSAL,
    "spkt_welch_density": L.FEAT_SPKT_WELCH,
    "large_standard_deviation": L.FEAT_LARGE_STD,
    "symmetry_looking": L.FEAT_SYMMETRY_LOOKING,
    "index_mass_quantile": L.FEAT_INDEX_MASS_QUANTILE,
    "longest_strike_above_mean": L.FEAT_LONGEST_STRIKE_ABOVE,
    "longest_strike_below_mean": L.FEAT_LONGEST_STRIKE_BELOW,
    "has_duplicate_max": L.FEAT_HAS_DUP_MAX,
    "has_duplicate_min": L.FEAT_HAS_DUP_MIN,
    "binned_entropy": L.FEAT_BINNED_ENTROPY,
    "mean_n_absolute_max": L.FEAT_MEAN_N_ABS_MAX,
    "benford_correlation": L.FEAT_BENFORD,
    "has_duplicate": L.FEAT_HAS_DUPLICATE,
    "percentage_of_reoccurring_datapoints_to_all_datapoints": L.FEAT_PCT_REOCCURRING_POINTS,
    "percentage_of_reoccurring_values_to_all_values": L.FEAT_PCT_REOCCURRING_VALUES,
    "sum_of_reoccurring_data_points": L.FEAT_SUM_REOCCURRING_POINTS,
    "sum_of_reoccurring_values": L.FEAT_SUM_REOCCURRING_VALUES,
    "ratio_value_number_to_time_series_length": L.FEAT_RATIO_UNIQUE_VALUES,
    "has_variance_larger_than_standard_deviation": L.FEAT_VAR_LARGER_THAN_STD,
    "count_value": L.FEAT_COUNT_VALUE,
    "partial_autocorrelation": L.FEAT_PARTIAL_AUTOCORRELATION,
    "spectral_frequency_ratio": L.FEAT_SPECTRAL_FREQ_RATIO,
    "fourier_entropy": L.FEAT_FOURIER_ENTROPY,
    "lempel_ziv_complexity": L.FEAT_LEMPEL_ZIV,
    "number_cwt_peaks": L.FEAT_NUMBER_CWT_PEAKS,
}

#: Features with several parameters (FCParameters keys as in the reference's
#: settings, src/pybasin/ts_torch/settings.py:263-346,407-417): name -> (defaults when
#: the config gives None, or None if the parameters are required).
FEATURE_MULTI: dict[str, list[dict[str, Any]] | None] = {
    "agg_autocorrelation": [{"f_agg": "mean", "maxlag": 40}],
    "energy_ratio_by_chunks": [{"num_segments": 10, "segment_focus": 0}],
    "count_in_range": None,
    "change_quantiles": None,
    "autocorrelation_periodicity": [{"output": "strength"}],
    "fft_aggregated": [{"aggtype": "centroid"}],
    "permutation_entropy": [{"tau": 1, "dimension": 3}],
    "agg_linear_trend": [{"attr": "slope", "chunk_size": 10, "f_agg": "mean"}],
    "ar_coefficient": [{"coeff": 0, "k": 1}],
    "cwt_coefficients": [{"widths": (2,), "coeff": 0, "w": 2}],
    "friedrich_coefficients": [{"coeff": 0, "m": 3, "r": 30}],
    "max_langevin_fixed_point": [{"m": 3, "r": 30}],
    "correlation_dimension": [{"emb_dim": 4, "lag": 1, "n_rvals": 50}],
    "lyapunov_r": [{"emb_dim": 10, "lag": 1, "trajectory_len": 20, "tau": 1.0}],
}
_AGG_ACF_KIND = {"mean": L.FEAT_AGG_AUTOCORR_MEAN, "median": L.FEAT_AGG_AUTOCORR_MEDIAN,
                 "var": L.FEAT_AGG_AUTOCORR_VAR}
_CHANGE_Q_KIND = {(False, "mean"): L.FEAT_CHANGE_QUANTILES_MEAN, (False, "var"): L.FEAT_CHANGE_QUANTILES_VAR,
                  (True, "mean"): L.FEAT_CHANGE_QUANTILES_ABS_MEAN, (True, "var"): L.FEAT_CHANGE_QUANTILES_ABS_VAR}


def _multi_column(fname: str, p: dict[str, Any], state: int) -> FeatureColumn:
    """One column of a multi-parameter feature: its kind and the (param, param2) pair."""
    name = _format_name(fname, p, state)
    if fname == "agg_autocorrelation":  # torch_features_autocorrelation.py:72-97
        f_agg = p.get("f_agg", "mean")
        if f_agg not in _AGG_ACF_KIND:
            raise ValueError(f"agg_autocorrelation: f_agg must be one of {sorted(_AGG_ACF_KIND)}, got {f_agg!r}")
        return FeatureColumn(state, _AGG_ACF_KIND[f_agg], float(p.get("maxlag", 40)), name)
    if fname == "energy_ratio_by_chunks":  # torch_features_advanced.py:93-105
        return FeatureColumn(state, L.FEAT_ENERGY_RATIO_BY_CHUNKS, float(p.get("num_segments", 10)), name,
                             float(p.get("segment_focus", 0)))
    if fname == "autocorrelation_periodicity":  # torch_features_autocorrelation.py:268-329
        out = p.get("output", "strength")
        kinds = {"strength": L.FEAT_ACF_PERIOD_STRENGTH, "period": L.FEAT_ACF_PERIOD_LAG}
        if out not in kinds:
            raise ValueError(f"autocorrelation_periodicity: output must be 'strength' or 'period', got {out!r}")
        return FeatureColumn(state, kinds[out], float(p.get("min_lag", 2)), name, float(p.get("peak_threshold", 0.3)))
    if fname == "fft_aggregated":  # torch_features_frequency.py:32-54
        agg = p.get("aggtype", "centroid")
        kinds = {"centroid": L.FEAT_FFT_AGG_CENTROID, "variance": L.FEAT_FFT_AGG_VARIANCE,
                 "skew": L.FEAT_FFT_AGG_SKEW, "kurtosis": L.FEAT_FFT_AGG_KURTOSIS}
        if agg not in kinds:
            raise ValueError(f"fft_aggregated: aggtype must be one of {sorted(kinds)}, got {agg!r}")
        return FeatureColumn(state, kinds[agg], 0.0, name)
    if fname == "permutation_entropy":  # torch_features_entropy_complexity.py:13-54
        return FeatureColumn(state, L.FEAT_PERMUTATION_ENTROPY, float(p.get("tau", 1)), name,
                             float(p.get("dimension", 3)))
    if fname == "agg_linear_trend":  # torch_features_trend.py:60-83
        kinds = {"mean": L.FEAT_AGG_TREND_MEAN, "var": L.FEAT_AGG_TREND_VAR, "min": L.FEAT_AGG_TREND_MIN,
                 "max": L.FEAT_AGG_TREND_MAX}
        f_agg, attr = p.get("f_agg", "mean"), p.get("attr", "slope")
        if f_agg not in kinds or attr not in _TREND_ATTRS:
            raise ValueError(f"agg_linear_trend: f_agg in {sorted(kinds)}, attr in {_TREND_ATTRS}; got {f_agg!r}, {attr!r}")
        return FeatureColumn(state, kinds[f_agg], float(p.get("chunk_size", 10)), name,
                             float(_TREND_ATTRS.index(attr)))
    if fname == "ar_coefficient":  # torch_features_trend.py:86-131
        return FeatureColumn(state, L.FEAT_AR_COEFFICIENT, float(p.get("k", 1)), name, float(p.get("coeff", 0)))
    if fname == "cwt_coefficients":  # torch_features_frequency.py:71-127
        w = int(p.get("w", 2))
        widths = tuple(int(v) for v in p.get("widths", (2,)))
        return FeatureColumn(state, L.FEAT_CWT, float(w), name, float(p.get("coeff", 0)) if w in widths else -1.0)
    if fname in ("friedrich_coefficients", "max_langevin_fixed_point"):  # torch_features_dynamical.py:87-174
        m_deg = int(p.get("m", 3))
        if not 0 <= m_deg <= 6:
            raise ValueError(f"{fname}: the fused fit takes polynomial degrees m <= 6, got {m_deg}")
        if fname == "friedrich_coefficients":
            return FeatureColumn(state, L.FEAT_FRIEDRICH, float(m_deg), name, float(p.get("coeff", 0)))
        return FeatureColumn(state, L.FEAT_LANGEVIN, float(m_deg), name)
    if fname == "correlation_dimension":  # ts_torch/torch_corr_dim.py:17-110
        emb, lag, nr = int(p.get("emb_dim", 4)), int(p.get("lag", 1)), int(p.get("n_rvals", 50))
        if not (1 <= emb <= 16 and 1 <= lag <= 100000 and 1 <= nr <= 1023):
            raise ValueError("correlation_dimension: emb_dim <= 16, lag <= 100000 and n_rvals <= 1023 are fused")
        return FeatureColumn(state, L.FEAT_CORR_DIM, float(emb), name, float(lag * 1024 + nr))
    if fname == "lyapunov_r":  # ts_torch/torch_lyapunov_r.py (Rosenstein)
        emb, lag, tl = int(p.get("emb_dim", 10)), int(p.get("lag", 1)), int(p.get("trajectory_len", 20))
        if float(p.get("tau", 1.0)) != 1.0 or not (1 <= emb <= 64 and 1 <= lag <= 100000 and 1 <= tl <= 1023):
            raise ValueError("lyapunov_r: the fused path takes tau = 1, emb_dim <= 64, trajectory_len <= 1023")
        return FeatureColumn(state, L.FEAT_LYAP_R, float(emb * 1024 + tl), name, float(lag))
    if fname == "count_in_range":  # torch_features_count.py:37-39
        return FeatureColumn(state, L.FEAT_COUNT_IN_RANGE, float(p["min_val"]), name, float(p["max_val"]))
    # change_quantiles, torch_features_change.py:113-140
    key = (bool(p.get("isabs", True)), p.get("f_agg", "mean"))
    if key not in _CHANGE_Q_KIND:
        raise ValueError(f"change_quantiles: f_agg must be 'mean' or 'var', got {key[1]!r}")
    return FeatureColumn(state, _CHANGE_Q_KIND[key], float(p["ql"]), name, float(p["qh"]))

#: Features whose ``attr`` parameter selects the kernel kind: name -> (kinds by
#: attr, default attr, numeric parameter key or None, its default).
FEATURE_ATTR: dict[str, tuple[dict[str, int], str, str | None, float]] = {
    "fft_coefficient": ({"real": L.FEAT_FFT_REAL, "imag": L.FEAT_FFT_IMAG, "abs": L.FEAT_FFT_ABS,
                         "angle": L.FEAT_FFT_ANGLE}, "abs", "coeff", 0.0),
    "linear_trend": ({"slope": L.FEAT_TREND_SLOPE, "intercept": L.FEAT_TREND_INTERCEPT,
                      "rvalue": L.FEAT_TREND_RVALUE, "pvalue": L.FEAT_TREND_PVALUE,
                      "stderr": L.FEAT_TREND_STDERR}, "slope", None, 0.0),
    "augmented_dickey_fuller": ({"teststat": L.FEAT_ADF_TESTSTAT, "pvalue": L.FEAT_ADF_PVALUE,
                                 "usedlag": L.FEAT_ADF_USEDLAG}, "teststat", None, 0.0),
    # the reference's linear_trend_timewise is linear_trend (torch_features_trend.py:54-56)
    "linear_trend_timewise": ({"slope": L.FEAT_TREND_SLOPE, "intercept": L.FEAT_TREND_INTERCEPT,
                               "rvalue": L.FEAT_TREND_RVALUE, "pvalue": L.FEAT_TREND_PVALUE,
                               "stderr": L.FEAT_TREND_STDERR}, "slope", None, 0.0),
}
_TREND_ATTRS = ("slope", "intercept", "rvalue", "pvalue", "stderr")

#: The parameter of each parameterised feature (its FCParameters key) and default.
FEATURE_PARAM: dict[int, tuple[str, float]] = {
    L.FEAT_CROSSINGS: ("m", 0.0),
    L.FEAT_QUANTILE: ("q", 0.5),
    L.FEAT_COUNT_ABOVE: ("t", 0.0),
    L.FEAT_COUNT_BELOW: ("t", 0.0),
    L.FEAT_NUMBER_PEAKS: ("n", 1.0),
    L.FEAT_AUTOCORRELATION: ("lag", 1.0),
    L.FEAT_RATIO_BEYOND_R_SIGMA: ("r", 1.0),
    L.FEAT_CID_CE: ("normalize", 1.0),
    L.FEAT_C3: ("lag", 1.0),
    L.FEAT_TIME_REVERSAL: ("lag", 1.0),
    L.FEAT_SPKT_WELCH: ("coeff", 2.0),
    L.FEAT_LARGE_STD: ("r", 0.25),
    L.FEAT_SYMMETRY_LOOKING: ("r", 0.1),
    L.FEAT_INDEX_MASS_QUANTILE: ("q", 0.5),
    L.FEAT_BINNED_ENTROPY: ("max_bins", 10.0),
    L.FEAT_MEAN_N_ABS_MAX: ("number_of_maxima", 1.0),
    L.FEAT_COUNT_VALUE: ("value", 0.0),
    L.FEAT_PARTIAL_AUTOCORRELATION: ("lag", 1.0),
    L.FEAT_FOURIER_ENTROPY: ("bins", 10.0),
    L.FEAT_LEMPEL_ZIV: ("bins", 2.0),
    L.FEAT_NUMBER_CWT_PEAKS: ("max_width", 5.0),
}

#: The reference's minimal set (src/pybasin/ts_torch/settings.py:376-395).
MINIMAL_FEATURES: dict[str, Any] = dict.fromkeys(
    [
        "median",
        "mean",
        "standard_deviation",
        "variance",
        "root_mean_square",
        "maximum",
        "absolute_maximum",
        "minimum",
        "delta",
        "log_delta",
    ]
)

DEFAULT_STEADY_FRACTION = 0.85  # src/pybasin/constants.py


def _format_name(base: str, params: dict[str, Any] | None, state: int) -> str:
    parts = [base]
    if params:
        parts.append("__".join(f"{k}_{v}" for k, v in sorted(params.items())))
    return f"state_{state}__" + "__".join(parts)


def columns_for(config: dict[str, Any] | None, state: int) -> list[FeatureColumn]:
    """Output columns for one state's FCParameters-style config, in config order."""
    cols: list[FeatureColumn] = []
    if not config:
        return cols
    for fname, plist in config.items():
        if fname in FEATURE_MULTI:
            defaults = FEATURE_MULTI[fname]
            if plist is None and defaults is None:
                raise ValueError(f"feature '{fname}' needs its parameters")
            cols.extend(_multi_column(fname, p, state) for p in (plist if plist is not None else defaults))
            continue
        if fname in FEATURE_ATTR:
            kinds, default_attr, key, default = FEATURE_ATTR[fname]
            for p in plist or [{"attr": default_attr, **({key: default} if key else {})}]:
                attr = p.get("attr", default_attr)
                if attr not in kinds:
                    raise ValueError(f"feature '{fname}': attr must be one of {sorted(kinds)}, got {attr!r}")
                value = float(p[key]) if key and key in p else default
                cols.append(FeatureColumn(state, kinds[attr], value, _format_name(fname, p, state)))
            continue
        if fname not in FEATURE_KINDS:
            raise ValueError(
                f"feature '{fname}' is not one of the fused statistics "
                f"{sorted([*FEATURE_KINDS, *FEATURE_ATTR, *FEATURE_MULTI])}; "
                "use B200Dopri5Solver(output='full') with the reference TorchFeatureExtractor for other features"
            )
        kind = FEATURE_KINDS[fname]
        if kind in FEATURE_PARAM:
            key, default = FEATURE_PARAM[kind]
            for p in plist or [{key: default}]:
                v = p[key]
                cols.append(FeatureColumn(state, kind, float(bool(v)) if isinstance(v, bool) else float(v),
                                          _format_name(fname, p, state)))
        else:
            if plist is not None:
                raise ValueError(f"feature '{fname}' takes no parameters")
            cols.append(FeatureColumn(state, kind, 0.0, _format_name(fname, None, state)))
    return cols


def impute_extreme(features: torch.Tensor, extreme_value: float = 1e10) -> torch.Tensor:
    """+inf -> +extreme, -inf -> -extreme, NaN -> +extreme (torch_feature_utilities.py:60-94)."""
    out = torch.nan_to_num(features, nan=extreme_value, posinf=extreme_value, neginf=-extreme_value)
    return out


class FusedFeatureExtractor:
    """Reference ``TorchFeatureExtractor`` API over features fused into the solver kernel."""

    def __init__(
        self,
        time_steady: float | None = None,
        features: str | dict[str, Any] | None = "minimal",
        features_per_state: dict[int, dict[str, Any] | None] | None = None,
        normalize: bool = True,
        device: str = "gpu",
        n_jobs: int | None = None,
        impute_method: str = "extreme",
    ):
        if impute_method != "extreme":
            raise ValueError("FusedFeatureExtractor supports impute_method='extreme' only")
        self.time_steady = time_steady
        if features in ("minimal", "comprehensive"):
            # 'comprehensive' spans FFT/entropy/... features that are not fused;
            # the fused kernel offers the minimal set for it.
            self.features: dict[str, Any] | None = dict(MINIMAL_FEATURES)
        else:
            self.features = features  # type: ignore[assignment]
        self.features_per_state = features_per_state or {}
        self.normalize = normalize
        self.device = device
        self.n_jobs = n_jobs
        self.impute_method = impute_method
        self._fit_lock = threading.Lock()
        self._is_fitted = False
        self._feature_mean: torch.Tensor | None = None
        self._feature_std: torch.Tensor | None = None
        self._extracted_feature_names: list[str] | None = None

    # -- configuration consumed by the solver ---------------------------------
    def columns(self, num_states: int) -> list[FeatureColumn]:
        cols: list[FeatureColumn] = []
        for s in range(num_states):
            if s in self.features_per_state:
                cfg = self.features_per_state[s]
                if cfg is not None:
                    cols += columns_for(cfg, s)
            elif self.features is not None:
                cols += columns_for(self.features, s)
        return cols

    def resolve_time_steady(self, save_ts: torch.Tensor) -> float:
        if self.time_steady is not None:
            return float(self.time_steady)
        t0, t1 = float(save_ts[0]), float(save_ts[-1])
        return t0 + DEFAULT_STEADY_FRACTION * (t1 - t0)

    # -- reference FeatureExtractor API ---------------------------------------
    def extract_features(self, solution: Any) -> torch.Tensor:
        y = solution.y
        feats: torch.Tensor | None = getattr(y, "_pb_features", None)
        names: list[str] | None = getattr(y, "_pb_feature_names", None)
        if feats is None or names is None:
            raise RuntimeError(
                "FusedFeatureExtractor reads features computed inside B200Dopri5Solver; construct the solver "
                "with feature_extractor=<this extractor> and pass its output solution"
            )
        self._extracted_feature_names = list(names)
        if feats.shape[1] == 0:
            return feats
        features = impute_extreme(feats)
        if self.normalize:
            with self._fit_lock:
                if not self._is_fitted:
                    self._feature_mean = features.mean(dim=0, keepdim=True)
                    std = features.std(dim=0, keepdim=True)
                    self._feature_std = torch.where(std == 0, torch.ones_like(std), std)
                    self._is_fitted = True
            assert self._feature_mean is not None and self._feature_std is not None
            features = (features - self._feature_mean.to(features.device)) / self._feature_std.to(features.device)
        return features

    def reset_scaler(self) -> None:
        with self._fit_lock:
            self._feature_mean = None
            self._feature_std = None
            self._is_fitted = False

    @property
    def feature_names(self) -> list[str]:
        if self._extracted_feature_names is None:
            raise RuntimeError("Feature names not available. Call extract_features first.")
        return self._extracted_feature_names


class FrictionFeatureExtractor:
    """The friction case study's extractor (case_studies/friction/friction_feature_extractor.py
    :17-41): one-hot [FP, LC] from max |y_1| over the window (FP if <= 0.2), with the
    maximum computed inside the integrator (``PB_FEAT_ABSMAX``)."""

    def __init__(self, time_steady: float | None = None, state: int = 1, threshold: float = 0.2,
                 device: str | torch.device = "cpu"):
        self.time_steady = time_steady
        self.state = state
        self.threshold = threshold
        self.device = device
        self.normalize = False

    def columns(self, num_states: int) -> list[FeatureColumn]:
        if not 0 <= self.state < num_states:
            raise ValueError(f"state {self.state} outside the {num_states}-dim system")
        return [FeatureColumn(self.state, L.FEAT_ABSMAX, 0.0, f"state_{self.state}__absolute_maximum")]

    def resolve_time_steady(self, save_ts: torch.Tensor) -> float:
        if self.time_steady is not None:
            return float(self.time_steady)
        t0, t1 = float(save_ts[0]), float(save_ts[-1])
        return t0 + DEFAULT_STEADY_FRACTION * (t1 - t0)

    def extract_features(self, solution: Any) -> torch.Tensor:
        feats = getattr(solution.y, "_pb_features", None)
        if feats is None:
            raise RuntimeError("FrictionFeatureExtractor reads features computed inside B200Dopri5Solver")
        lc = (feats[:, 0] > self.threshold).to(torch.float64)
        return torch.stack([1.0 - lc, lc], dim=1)

    @property
    def feature_names(self) -> list[str]:
        return ["FP", "LC"]
