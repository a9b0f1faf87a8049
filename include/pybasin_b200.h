/*
 * pybasin_b200 — C ABI of the B200 fused Dopri5 + steady-state-feature library.
 *
 * Every entry point takes plain pointers and sizes.  Array arguments marked
 * "device" are CUDA device pointers on the current device; `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).  No entry point
 * allocates on the caller's behalf except where stated, none aborts, and every
 * one returns a pb_status (0 = success, negative = error, the numbering of the
 * reference's native solver ABI extended with a few codes).
 *
 * Reference interfaces replaced (paths relative to the pybasin project root):
 *   pb_solve_batch      src/zigode/src/c_api.zig:193-314 (`solve_batch`) and the
 *                       Python-level SolverProtocol.integrate it backs,
 *                       src/pybasin/protocols.py:156-168,
 *                       src/pybasin/solvers/torchdiffeq_solver.py:97-134;
 *                       fused with TorchFeatureExtractor.extract_features,
 *                       src/pybasin/ts_torch/torch_feature_extractor.py:192-287.
 *   pb_label_nearest    the 1-NN classification + basin-stability count step,
 *                       src/pybasin/basin_stability_estimator.py:426-446,586-598
 *                       (sklearn KNeighborsClassifier(n_neighbors=1) predict).
 *   pb_error_string     src/zigode/zig_solver.py:333-341 (error-code messages).
 */
#ifndef PYBASIN_B200_H
#define PYBASIN_B200_H

#ifndef __CUDACC_RTC__
#include <stdint.h> /* under NVRTC the including kernel header supplies the fixed-width types */
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes (0/-1/-2/-3 as in src/zigode/src/c_api.zig:17-23) ---- */
typedef enum {
    PB_SUCCESS = 0,
    PB_EINVALID_ODE = -1,   /* unknown system id / dimension combination */
    PB_EALLOC = -2,         /* device allocation failed */
    PB_ESOLVE = -3,         /* kernel launch or execution error */
    PB_EINVAL = -5,         /* invalid argument (null pointer, bad size, bad layout) */
    PB_ECUDA = -6,          /* other CUDA runtime error */
    PB_EUNSUPPORTED = -7,   /* valid request the library does not support (e.g. a kernel variant not compiled in) */
    PB_ECOMPILE = -8,       /* runtime (NVRTC) compilation of a user right-hand side failed */
    PB_ESCRATCH_LIMIT = -9  /* pb_solve_batch_noalloc: request needs more than PB_NOALLOC_SCRATCH_BYTES */
} pb_status;

/* ---- built-in right-hand sides (templated device functors) ---- */
typedef enum {
    PB_SYS_LINEAR = 0,        /* dy/dt = p0*y, any dim 1..4; tests/unit/solvers/test_solver.py:16-21 */
    PB_SYS_PENDULUM = 1,      /* case_studies/pendulum/pendulum_ode.py:23-40, p=[alpha,T,K] */
    PB_SYS_DUFFING = 2,       /* case_studies/duffing_oscillator/duffing_ode.py:26-42, p=[delta,k3,A] */
    PB_SYS_LORENZ = 3,        /* case_studies/lorenz/lorenz_jax_ode.py, p=[sigma,r,b] */
    PB_SYS_LORENZ_MASKED = 4, /* case_studies/lorenz/lorenz_ode.py:28-64 (|y|>=200 freezes) */
    PB_SYS_ROSSLER_NET = 5,   /* case_studies/rossler_network/rossler_network_jax_ode.py:53-79 */
    PB_SYS_FRICTION = 6,      /* case_studies/friction/friction_ode.py:32-75, p=[v_d,xi,musd,mud,muv,v0] */
    PB_SYS_USER = 64          /* a right-hand side compiled at run time (pb_rhs_compile),
                                 solved with pb_solve_batch_rhs */
} pb_system;

/* ---- arithmetic of the integrator ---- */
typedef enum {
    PB_PREC_FP64 = 0,  /* plain: stages, state, time, error norm and control all FP64 */
    PB_PREC_MIXED = 1  /* FP32 stages and state (Kahan-compensated accumulation),
                          FP64 time, error norm and step-size control */
} pb_precision;

/* ---- how trajectories map to initial conditions and parameter rows ---- */
typedef enum {
    PB_LAYOUT_SINGLE = 0,  /* every trajectory uses params row 0; traj j uses y0 row j */
    PB_LAYOUT_CROSS = 1,   /* IC-major product, src/pybasin/solvers/base.py:155-159:
                              traj j = ic*P + p uses y0 row ic and params row p */
    PB_LAYOUT_INDEXED = 2  /* traj j uses y0 row j and params row param_index[j] */
} pb_layout;

/* ---- fused window features (names of src/pybasin/ts_torch/settings.py) ---- */
typedef enum {
    PB_FEAT_MEDIAN = 0, PB_FEAT_MEAN = 1, PB_FEAT_STD = 2, PB_FEAT_VAR = 3, PB_FEAT_RMS = 4,
    PB_FEAT_MAX = 5, PB_FEAT_ABSMAX = 6, PB_FEAT_MIN = 7, PB_FEAT_DELTA = 8,
    PB_FEAT_LOG_DELTA = 9, PB_FEAT_AMPLITUDE = 10, PB_FEAT_CROSSINGS = 11, PB_FEAT_LAST = 12,
    /* network systems: max - min over the nodes of block feat_state (0 x, 1 y, 2 z;
       3 = the largest of the three) at t1, the synchronisation features of
       case_studies/rossler_network/synchronization_feature_extractor.py:73-106 */
    PB_FEAT_SYNC_DEV = 13,
    /* wider set, streaming (ts_torch/calculators/torch_features_statistical.py:20-27,
       119-122,160-163 and :50-57 for length) */
    PB_FEAT_SUM = 14, PB_FEAT_ABS_ENERGY = 15, PB_FEAT_LENGTH = 16, PB_FEAT_VARIATION_COEFF = 17,
    /* wider set from the stored window (a second pass; feat_param as noted):
       quantile (q, torch.quantile linear), kurtosis, skewness (statistical.py:125-156),
       absolute_sum_of_changes, mean_abs_change, mean_change, mean_second_derivative_central
       (torch_features_change.py:79-110), count_above_mean, count_below_mean, count_above (t),
       count_below (t) (torch_features_count.py:11-33), number_peaks (n, pattern.py:64-110),
       autocorrelation (lag, torch_features_autocorrelation.py:13-27),
       ratio_beyond_r_sigma (r, statistical.py:176-182) */
    PB_FEAT_QUANTILE = 18, PB_FEAT_KURTOSIS = 19, PB_FEAT_SKEWNESS = 20, PB_FEAT_ABS_SUM_CHANGES = 21,
    PB_FEAT_MEAN_ABS_CHANGE = 22, PB_FEAT_MEAN_CHANGE = 23, PB_FEAT_MEAN_SECOND_DERIV = 24,
    PB_FEAT_COUNT_ABOVE_MEAN = 25, PB_FEAT_COUNT_BELOW_MEAN = 26, PB_FEAT_COUNT_ABOVE = 27,
    PB_FEAT_COUNT_BELOW = 28, PB_FEAT_NUMBER_PEAKS = 29, PB_FEAT_AUTOCORRELATION = 30,
    PB_FEAT_RATIO_BEYOND_R_SIGMA = 31,
    /* fft_coefficient (coeff = feat_param; the attribute in the kind: real, imag,
       abs, angle; torch_features_frequency.py:11-29), linear_trend (the attribute
       in the kind; torch_features_trend.py:11-51), first/last location of the
       maximum/minimum (torch_features_location.py:11-49), cid_ce (normalize =
       feat_param 0/1; torch_features_entropy_complexity.py:182-190), c3 (lag) and
       time_reversal_asymmetry_statistic (lag) (torch_features_advanced.py:84-90,
       109-118) */
    PB_FEAT_FFT_REAL = 32, PB_FEAT_FFT_IMAG = 33, PB_FEAT_FFT_ABS = 34, PB_FEAT_FFT_ANGLE = 35,
    PB_FEAT_TREND_SLOPE = 36, PB_FEAT_TREND_INTERCEPT = 37, PB_FEAT_TREND_RVALUE = 38,
    PB_FEAT_TREND_PVALUE = 39, PB_FEAT_TREND_STDERR = 40,
    PB_FEAT_FIRST_LOC_MAX = 41, PB_FEAT_FIRST_LOC_MIN = 42, PB_FEAT_LAST_LOC_MAX = 43,
    PB_FEAT_LAST_LOC_MIN = 44, PB_FEAT_CID_CE = 45, PB_FEAT_C3 = 46, PB_FEAT_TIME_REVERSAL = 47,
    /* spkt_welch_density (coeff; torch_features_frequency.py:57-65),
       large_standard_deviation (r; torch_features_boolean.py:44-48), symmetry_looking
       (r; torch_features_statistical.py:185-191), index_mass_quantile (q;
       torch_features_location.py:52-65), longest_strike_above_mean /
       longest_strike_below_mean (torch_features_pattern.py:10-53) */
    PB_FEAT_SPKT_WELCH = 48, PB_FEAT_LARGE_STD = 49, PB_FEAT_SYMMETRY_LOOKING = 50,
    PB_FEAT_INDEX_MASS_QUANTILE = 51, PB_FEAT_LONGEST_STRIKE_ABOVE = 52, PB_FEAT_LONGEST_STRIKE_BELOW = 53,
    /* has_duplicate_max / has_duplicate_min (torch_features_boolean.py:23-34),
       binned_entropy (max_bins <= 256; torch_features_entropy_complexity.py:58-100),
       mean_n_absolute_max (number_of_maxima <= 64; torch_features_statistical.py:166-172),
       benford_correlation (torch_features_advanced.py:21-81) */
    PB_FEAT_HAS_DUP_MAX = 54, PB_FEAT_HAS_DUP_MIN = 55, PB_FEAT_BINNED_ENTROPY = 56,
    PB_FEAT_MEAN_N_ABS_MAX = 57, PB_FEAT_BENFORD = 58,
    /* repeated values over the whole window, from the sorted window (at most
       PB_SORTED_WINDOW_MAX samples): has_duplicate (torch_features_boolean.py:11-20),
       percentage_of_reoccurring_datapoints_to_all_datapoints, percentage_of_reoccurring_
       values_to_all_values, sum_of_reoccurring_data_points, sum_of_reoccurring_values,
       ratio_value_number_to_time_series_length (torch_features_reocurrance.py:10-163);
       then has_variance_larger_than_standard_deviation (torch_features_boolean.py:37-41)
       and count_value (value, compared in FP32 like the stored window;
       torch_features_count.py:42-45) */
    PB_FEAT_HAS_DUPLICATE = 59, PB_FEAT_PCT_REOCCURRING_POINTS = 60, PB_FEAT_PCT_REOCCURRING_VALUES = 61,
    PB_FEAT_SUM_REOCCURRING_POINTS = 62, PB_FEAT_SUM_REOCCURRING_VALUES = 63, PB_FEAT_RATIO_UNIQUE_VALUES = 64,
    PB_FEAT_VAR_LARGER_THAN_STD = 65, PB_FEAT_COUNT_VALUE = 66,
    /* partial_autocorrelation (lag <= 64; Durbin-Levinson,
       torch_features_autocorrelation.py:31-68), agg_autocorrelation over lags
       1..maxlag (maxlag <= 128; f_agg mean / median / var in the kind,
       torch_features_autocorrelation.py:72-97), energy_ratio_by_chunks
       (num_segments, feat_param2 = segment_focus; torch_features_advanced.py:93-105),
       count_in_range (min_val, feat_param2 = max_val, compared in FP32 like the
       stored window; torch_features_count.py:37-39), change_quantiles (ql,
       feat_param2 = qh; isabs and f_agg in the kind; torch_features_change.py:20-75,
       113-140) */
    PB_FEAT_PARTIAL_AUTOCORRELATION = 67, PB_FEAT_AGG_AUTOCORR_MEAN = 68, PB_FEAT_AGG_AUTOCORR_MEDIAN = 69,
    PB_FEAT_AGG_AUTOCORR_VAR = 70, PB_FEAT_ENERGY_RATIO_BY_CHUNKS = 71, PB_FEAT_COUNT_IN_RANGE = 72,
    PB_FEAT_CHANGE_QUANTILES_MEAN = 73, PB_FEAT_CHANGE_QUANTILES_VAR = 74,
    PB_FEAT_CHANGE_QUANTILES_ABS_MEAN = 75, PB_FEAT_CHANGE_QUANTILES_ABS_VAR = 76,
    /* autocorrelation_periodicity (min_lag, feat_param2 = peak_threshold; output
       strength / period in the kind; torch_features_autocorrelation.py:268-329, peaks
       as torch_feature_utilities.py:146-218) */
    PB_FEAT_ACF_PERIOD_STRENGTH = 77, PB_FEAT_ACF_PERIOD_LAG = 78,
    /* from the window's power spectrum (at most PB_SPECTRAL_WINDOW_MAX samples):
       spectral_frequency_ratio (torch_features_frequency.py:390-441) and
       fft_aggregated with aggtype centroid / variance / skew / kurtosis in the kind
       (torch_features_frequency.py:32-54) */
    PB_FEAT_SPECTRAL_FREQ_RATIO = 79, PB_FEAT_FFT_AGG_CENTROID = 80, PB_FEAT_FFT_AGG_VARIANCE = 81,
    PB_FEAT_FFT_AGG_SKEW = 82, PB_FEAT_FFT_AGG_KURTOSIS = 83,
    /* fourier_entropy (bins, unused as in the reference; a spectral kind;
       torch_features_entropy_complexity.py:97-110), permutation_entropy (tau,
       feat_param2 = dimension <= 7; :13-54), lempel_ziv_complexity (bins <= 255, at
       most PB_SYMBOLIC_WINDOW_MAX window samples; :141-178) */
    PB_FEAT_FOURIER_ENTROPY = 84, PB_FEAT_PERMUTATION_ENTROPY = 85, PB_FEAT_LEMPEL_ZIV = 86,
    /* agg_linear_trend (chunk_size, feat_param2 = attribute 0..4: slope, intercept,
       rvalue, pvalue, stderr; f_agg mean / var / min / max in the kind;
       torch_features_trend.py:60-83), ar_coefficient (k <= 10, feat_param2 = coeff;
       Yule-Walker, torch_features_trend.py:86-131) */
    PB_FEAT_AGG_TREND_MEAN = 87, PB_FEAT_AGG_TREND_VAR = 88, PB_FEAT_AGG_TREND_MIN = 89,
    PB_FEAT_AGG_TREND_MAX = 90, PB_FEAT_AR_COEFFICIENT = 91,
    /* cwt_coefficients (w, feat_param2 = coeff, -1 when w is not one of the widths;
       Ricker wavelet, torch_features_frequency.py:71-127), friedrich_coefficients
       (m <= 6, feat_param2 = coeff) and max_langevin_fixed_point (m <= 6)
       (torch_features_dynamical.py:87-174) */
    PB_FEAT_CWT = 92, PB_FEAT_FRIEDRICH = 93, PB_FEAT_LANGEVIN = 94,
    /* augmented_dickey_fuller with attr teststat / pvalue / usedlag in the kind
       (torch_features_trend.py:134-169), number_cwt_peaks (max_width <= 64;
       torch_features_pattern.py:154-188) */
    PB_FEAT_ADF_TESTSTAT = 95, PB_FEAT_ADF_PVALUE = 96, PB_FEAT_ADF_USEDLAG = 97, PB_FEAT_NUMBER_CWT_PEAKS = 98,
    /* correlation_dimension (emb_dim <= 16, feat_param2 = lag * 1024 + n_rvals with
       n_rvals <= 1023; Grassberger-Procaccia as src/pybasin/ts_torch/torch_corr_dim.py:17-110
       states it; a symbolic kind, at most PB_SPECTRAL_WINDOW_MAX window samples) */
    PB_FEAT_CORR_DIM = 99,
    /* lyapunov_r (feat_param = emb_dim * 1024 + trajectory_len, feat_param2 = lag, tau
       = 1; Rosenstein as src/pybasin/ts_torch/torch_lyapunov_r.py states it; a
       symbolic kind, at most PB_SPECTRAL_WINDOW_MAX window samples) */
    PB_FEAT_LYAP_R = 100
} pb_feature;
#define PB_FEAT_LAST_KIND PB_FEAT_LYAP_R
/* kinds computed from the stored feature window (PB_FEAT_MEDIAN and 18..100): the
   window costs n_traj x (n_save - win_begin) floats of scratch per such column */
#define PB_FEAT_IS_WINDOW(k) ((k) == PB_FEAT_MEDIAN || ((k) >= PB_FEAT_QUANTILE && (k) <= PB_FEAT_LAST_KIND))
/* kinds 59..64 sort the window in shared memory: a request with more window
   samples than this returns PB_EUNSUPPORTED */
#define PB_FEAT_IS_SORTED(k) ((k) >= PB_FEAT_HAS_DUPLICATE && (k) <= PB_FEAT_RATIO_UNIQUE_VALUES)
#define PB_SORTED_WINDOW_MAX 32768
/* kinds 79..84 hold the window's power spectrum in shared memory: a request with
   more window samples than this returns PB_EUNSUPPORTED */
#define PB_FEAT_IS_SPECTRAL(k) ((k) >= PB_FEAT_SPECTRAL_FREQ_RATIO && (k) <= PB_FEAT_FOURIER_ENTROPY)
#define PB_SPECTRAL_WINDOW_MAX 16384
/* kinds 85, 86, 99 and 100 run one block per column with their data in shared memory */
#define PB_FEAT_IS_SYMBOLIC(k) \
    ((k) == PB_FEAT_PERMUTATION_ENTROPY || (k) == PB_FEAT_LEMPEL_ZIV || (k) == PB_FEAT_CORR_DIM || (k) == PB_FEAT_LYAP_R)
#define PB_SYMBOLIC_WINDOW_MAX 8191

/* ---- per-trajectory status written to status_out ---- */
typedef enum {
    PB_TRAJ_OK = 0,
    PB_TRAJ_MAX_STEPS = 1,    /* max_steps attempted steps before t1 */
    PB_TRAJ_DT_UNDERFLOW = 2, /* t + dt == t */
    PB_TRAJ_UNBOUNDED = 3,    /* max|y| >= unbounded_threshold after an accepted step */
    PB_TRAJ_NONFINITE = 4,    /* non-finite error norm */
    PB_TRAJ_BAD_INPUT = 5     /* param_index row outside [0, n_param_rows) */
} pb_traj_status;

#define PB_MAX_FEATURES 32
#define PB_MAX_CROSSING 4
#define PB_MAX_PARAMS 8

typedef enum { PB_DTYPE_F32 = 0, PB_DTYPE_F64 = 1 } pb_dtype;

/* Work distribution of pb_solve_batch. */
typedef enum {
    PB_SCHED_PLAIN = 0,  /* one thread per trajectory, grid covers all trajectories */
    PB_SCHED_QUEUE = 1,  /* persistent lanes refilled from a global atomic queue with
                            warp-aggregated fetches (needs `queue_counter`) */
    PB_SCHED_PROBED = 2  /* the queue in predicted-cost order: every trajectory first
                            integrates the first 5 % of [t0, t1] (its step count there
                            predicts its total), the trajectories are sorted longest
                            first (stably, so `order` is kept within equal counts) and
                            resumed from their saved state; results are identical to
                            PB_SCHED_QUEUE.  Applies with deferred dense output; other
                            requests run as PB_SCHED_QUEUE.  Needs `queue_counter`. */
} pb_schedule;

typedef struct pb_solve_args {
    /* problem */
    int32_t system;          /* pb_system */
    int32_t dim;             /* state dimension S */
    int32_t precision;       /* pb_precision */
    int32_t schedule;        /* pb_schedule */
    int32_t layout;          /* pb_layout */
    int32_t y0_dtype;        /* pb_dtype of y0 */
    int32_t n_params;        /* columns of params (<= PB_MAX_PARAMS) */
    int32_t block_size;      /* threads per block (0 = library default: 64 queue, 128 plain) */
    int32_t grid_blocks;     /* QUEUE: persistent blocks (0 = occupancy-derived) */
    int32_t _pad0;
    int64_t n_ic;            /* rows of y0 */
    int64_t n_param_rows;    /* rows of params */
    int64_t n_traj;          /* trajectories to integrate */
    const void* y0;          /* device (n_ic, dim) */
    const double* params;    /* device (n_param_rows, n_params) */
    const int32_t* param_index; /* device (n_traj) for PB_LAYOUT_INDEXED, else NULL */
    const int32_t* csr_row;  /* device, network systems only: (n_nodes+1) */
    const int32_t* csr_col;  /* device, network systems only */
    /* time grid */
    double t0, t1;           /* integrate from t0 to t1 */
    const double* save_ts;   /* device (n_save) ascending save instants */
    int32_t n_save;
    int32_t win_begin;       /* first save index of the feature window */
    /* control */
    double rtol, atol;
    int64_t max_steps;       /* attempted steps per trajectory */
    double unbounded_thr;    /* <= 0 disables the stop-on-|y| event */
    /* features: output column c = feature feat_kind[c] of state feat_state[c] */
    int32_t n_features;
    int32_t _pad1;
    int32_t feat_state[PB_MAX_FEATURES];
    int32_t feat_kind[PB_MAX_FEATURES];
    double feat_param[PB_MAX_FEATURES]; /* level m of PB_FEAT_CROSSINGS */
    /* outputs (device; any may be NULL) */
    double* features_out;    /* (n_traj, n_features) */
    int32_t* status_out;     /* (n_traj) pb_traj_status */
    void* y_final_out;       /* (n_traj, dim) state at t1 (or at the stop) */
    void* y_full_out;        /* (n_save, n_traj, dim): every save point, reference layout */
    int32_t y_out_dtype;     /* pb_dtype of y_final_out / y_full_out */
    int32_t _pad2;
    int64_t* steps_out;      /* (n_traj) attempted steps */
    /* scratch (device) */
    unsigned long long* queue_counter; /* QUEUE schedule: one counter (the call resets it on `stream`) */
    void* scratch;           /* pb_solve_scratch_bytes(args) bytes, 256-byte aligned; NULL when that is 0 */
    /* processing order (device, optional): queue position q integrates trajectory
       order[q], a permutation of [0, n_traj) (entries outside that range are skipped).  Ordering ICs along a space-filling
       curve puts trajectories with similar dynamics (and step counts) in the same
       warp.  Outputs stay indexed by trajectory. */
    const int32_t* order;
    int32_t dense_mode;      /* pb_dense_mode */
    int32_t window_record_cap; /* PB_DENSE_DEFERRED: step records per trajectory (0 = default) */
    /* orbit data (utils.py:254-303 extract_orbit_data, torch_features_pattern.py:113-150
       extract_peak_values): for the p-th PB_FEAT_NUMBER_PEAKS column (in column
       order; its state and support n), the values of the strict local maxima of the
       window in time order, the first peak_cap of them, at
       peaks_out[(traj * n_peak_columns + p) * peak_cap + i], NaN-padded; the column
       itself holds the full count.  NULL = not written. */
    double* peaks_out;
    int32_t peak_cap;
    /* QUEUE / PROBED schedules (ABI >= 102): a warp fetches new queue positions for
       its idle lanes once refill_lanes of its 32 lanes are idle, so lanes whose
       trajectories finished early take new work (0 or 32: when all 32 are idle). */
    int32_t refill_lanes;
    /* second parameter of the two-parameter window kinds (segment_focus, max_val, qh) */
    double feat_param2[PB_MAX_FEATURES];
} pb_solve_args;

/* Where the save points of the feature window are evaluated. */
typedef enum {
    PB_DENSE_INLINE = 0,   /* by the integrating thread, right after each accepted step */
    PB_DENSE_DEFERRED = 1  /* two passes: the integrator writes one record (step start, step
                              size, interpolation coefficients of the feature states) per window
                              step that holds save points; a sampling kernel then evaluates all
                              save points of a trajectory across the lanes of one warp.  A
                              trajectory whose window needs more than window_record_cap records
                              is integrated again with the inline path.  Not combinable with
                              y_full_out (which uses the inline path). */
} pb_dense_mode;

/* Integrate n_traj trajectories with adaptive Dormand-Prince 5(4) and write the
 * fused window features, statuses and (optionally) states.  Asynchronous on
 * `stream`.  Replaces src/zigode/src/c_api.zig:193-314 (solve_batch) and
 * src/pybasin/solvers/torchdiffeq_solver.py:97-134 + the minimal statistics of
 * src/pybasin/ts_torch/calculators/torch_features_statistical.py. */
int pb_solve_batch(const pb_solve_args* args, void* stream);

/* Device bytes of `scratch` that pb_solve_batch needs for `args`: the median
 * windows (n_traj x median columns x window length floats) and, in
 * PB_DENSE_DEFERRED mode, the step records and per-trajectory record counts. */
int64_t pb_solve_scratch_bytes(const pb_solve_args* args);

/* 1-NN labelling on the device (Euclidean, the reference's
 * KNeighborsClassifier(n_neighbors=1), src/pybasin/basin_stability_estimator.py:426-446)
 * followed by per-group label counts (src/pybasin/basin_stability_estimator.py:586-598).
 *   features   device (n, n_features) double
 *   templates  device (n_templates, n_features) double
 *   tpl_label  device (n_templates) int32 class of each template (0..n_classes-1)
 *   status     device (n) int32 or NULL; PB_TRAJ_UNBOUNDED rows get class n_classes
 *   group_of   device (n) int32 or NULL (all rows group 0)
 *   labels_out device (n) int32
 *   counts_out device (n_groups, n_classes + 1) int64, zeroed by the call on `stream`
 * Non-finite features are imputed first (+inf,NaN -> +1e10, -inf -> -1e10),
 * src/pybasin/ts_torch/torch_feature_utilities.py:60-94. */
int pb_label_nearest(const double* features, int64_t n, int32_t n_features,
                     const double* templates, int32_t n_templates, const int32_t* tpl_label,
                     int32_t n_classes, const int32_t* status, const int32_t* group_of,
                     int32_t n_groups, int32_t* labels_out, int64_t* counts_out, void* stream);

/* Z-order (Morton) keys of the ICs over their bounding box: argsort of the keys
 * is the processing order passed as pb_solve_args.order (neighbouring ICs mostly
 * share an attractor and a step count, so a warp's lanes finish together).
 * No reference counterpart: the reference integrates in batch order.
 *   y0        device (n, dim) f32 or f64 (y0_dtype), row-major
 *   bits      bits per coordinate of the first min(dim, 4) coordinates, bits*min(dim,4) <= 62
 *   groups    optional device (n,) int32: keys become group-major (group << 40 | top 40 key bits)
 *   bbox_work device scratch of 8 uint64, overwritten on `stream`
 *   keys_out  device (n,) int64
 * NaN coordinates do not widen the bounding box and quantise to 0. */
int pb_morton_keys(const void* y0, int32_t y0_dtype, int64_t n, int32_t dim, int32_t bits,
                   const int32_t* groups, uint64_t* bbox_work, int64_t* keys_out, void* stream);
/* Processing order from keys: order_out (n int32) = the stable ascending argsort of
 * keys[0..n) on bits [0, end_bit) (an LSD radix sort; keys is clobbered).  scratch
 * holds pb_morton_order_scratch_bytes(n) bytes (256-byte aligned).  No reference
 * counterpart (see pb_morton_keys). */
int64_t pb_morton_order_scratch_bytes(int64_t n);
int pb_morton_order(int64_t* keys, int64_t n, int32_t end_bit, void* scratch, int64_t scratch_bytes,
                    int32_t* order_out, void* stream);

/* Occupancy helper for the autotuner: resident blocks per SM of the pb_solve_batch
 * kernel selected by (system, dim, precision, schedule) at `block_size`. */
int pb_query_occupancy(int32_t system, int32_t dim, int32_t precision, int32_t schedule,
                       int32_t block_size, int32_t* blocks_per_sm, int32_t* num_sms);

/* Throughput probe for the roofline denominator of the integrator kernels, whose
 * bound is the FP32 (mixed) or FP64 (plain) FMA pipe rather than HBM or the tensor
 * cores: launches `blocks` x 256 threads, each running `iters` x 8 independent
 * FMA chains in FP32 (precision PB_PREC_MIXED) or FP64 (PB_PREC_FP64), and writes
 * one value per thread to `sink` (device, blocks*256 floats) so nothing is elided.
 * The caller times it; flops = 2 * 8 * iters * blocks * 256.  No reference
 * counterpart (measurement utility). */
int pb_probe_fma(int32_t precision, int32_t blocks, int32_t iters, float* sink, void* stream);

/* Allocation-free variant of pb_solve_batch.  No counterpart in the reference:
 * it exists for callers that may not allocate device memory themselves, such as
 * plug-ins of a host application that owns all device memory under a fixed
 * budget, or latency-critical loops that cannot afford cudaMalloc.  The caller
 * still provides every input and output array; args->scratch and
 * args->queue_counter are ignored and replaced by a fixed array of
 * PB_NOALLOC_SCRATCH_BYTES bytes that this library reserves on every GPU it is
 * loaded on (held until the process exits).  A request whose scratch
 * (pb_solve_scratch_bytes + 256) exceeds that size returns PB_ESCRATCH_LIMIT and
 * launches nothing.  The first call on a device looks up the array's device
 * address (once per device and context: after cudaDeviceReset the next call
 * looks it up again); make that first call before any stream capture.
 * All calls on a device share the one array: calls whose kernels may overlap on
 * the GPU (different streams, or several host threads) race and must be
 * serialised by the caller.  The call itself allocates nothing. */
#define PB_NOALLOC_SCRATCH_BYTES (64ll * 1024ll * 1024ll)
int pb_solve_batch_noalloc(const pb_solve_args* args, void* stream);

/* ---- right-hand sides compiled at run time (NVRTC) -------------------------
 * Replaces the reference's SymPy-to-C path for user ODEs, src/zigode/sympy_ode.py
 * :49-78 (C source from symbolic expressions, compiled into a library that the
 * native solver loads, zig_solver.py:106-179).  Here the expressions become a
 * device functor inside the same fused integrator templates, compiled for
 * sm_100a by NVRTC (loaded with dlopen: libnvrtc.so.12 of the CUDA toolkit, or
 * the path in PB_NVRTC_LIBRARY).
 *   rhs          dim C expressions, dy[i]/dt = rhs[i], in terms of y[j] (state,
 *                stage precision), p[k] (parameters, stage precision) and t (FP64);
 *                math functions of CUDA device code (sin, cos, exp, pow, ...)
 *   dim          1..PB_MAX_USER_DIM;  n_params 0..PB_MAX_PARAMS
 *   preamble     optional device code placed before the functor (helper
 *                __device__ functions), or NULL
 *   precision    pb_precision of the kernels to build
 *   include_dirs directories holding pb_dopri5.cuh and pybasin_b200.h; with
 *                n_include_dirs = 0 they are found next to this library
 *                (../csrc and ../../include relative to its file)
 *   cache_dir    optional directory for compiled modules, keyed by a hash of the
 *                generated source and the compile options, or NULL
 *   out          receives the loaded program on the current device; with
 *                out = NULL the call only compiles (and fills cache_dir), which
 *                needs no GPU
 *   log          optional buffer for the NVRTC log (PB_ECOMPILE on a failed compile)
 * The program holds a module on the device that was current; release it with
 * pb_rhs_release. */
#define PB_MAX_USER_DIM 16
typedef struct pb_rhs_program pb_rhs_program;
int pb_rhs_compile(const char* const* rhs, int32_t dim, int32_t n_params, const char* preamble,
                   int32_t precision, const char* const* include_dirs, int32_t n_include_dirs,
                   const char* cache_dir, pb_rhs_program** out, char* log, int64_t log_bytes);
/* pb_solve_batch for a compiled right-hand side: args->system = PB_SYS_USER,
 * args->dim / precision / n_params equal to the program's; every other field as
 * for pb_solve_batch (features on states < 8). */
int pb_solve_batch_rhs(const pb_rhs_program* prog, const pb_solve_args* args, void* stream);
int pb_rhs_release(pb_rhs_program* prog);

/* ---- learned surrogate (no counterpart in the reference) -------------------
 * A small MLP maps (initial condition, parameters) to attractor-class logits;
 * it is trained on labels produced by pb_solve_batch + pb_label_nearest, and its
 * low-confidence predictions (plus an audited random slice) are integrated.
 * BF16 operands, FP32 accumulation (mma.sync m16n8k16), all arrays device. */

/* C[m,n] = alpha * sum_k A(m,k) B(k,n) (+ bias[n]), optionally GELU; A(m,k) is
 * A[m*sam + k*sak], B(k,n) is B[k*sbk + n*sbn] (BF16).  Outputs (row stride ldc):
 * c_f32 (FP32), c_bf16 (BF16), z_pre (FP32 value before the activation); any may
 * be NULL but not all. */
int pb_mlp_gemm(const void* A, int64_t sam, int64_t sak, const void* B, int64_t sbk, int64_t sbn,
                const float* bias, float alpha, int32_t M, int32_t N, int32_t K, int32_t gelu,
                float* c_f32, void* c_bf16, float* z_pre, int64_t ldc, void* stream);
/* MLP inference on the 5th-generation tensor cores (tcgen05.mma, FP32
 * accumulators in tensor memory): the whole network for 128 rows per CTA, the
 * activations kept in shared memory between layers, GELU after every layer but
 * the last.  x: device (n, d_in) BF16.  Layer l has n_pad[l] x k_pad[l] weights
 * (multiples of 16, <= 256, k_pad[l] = n_pad[l-1], k_pad[0] >= d_in) packed in
 * the MMA operand layout (8 x 8 BF16 core matrices, core (n/8, k/8) at
 * ((n/8)*(k_pad/8) + k/8) * 128 bytes, rows of a core 16 bytes apart; zero
 * padding), 16-byte aligned, and n_real[l] biases (FP32).  w_packed, bias,
 * n_pad, k_pad, n_real are host arrays of n_layers entries (<= 8).  logits:
 * device (n, n_classes) FP32.  error_flag (device int32, optional) is set to 1
 * if a CTA gave up waiting on its tensor-core or copy completion. */
int pb_mlp_infer_tc(const void* x_bf16, int64_t n, int32_t d_in, int32_t n_layers,
                    const void* const* w_packed, const float* const* bias, const int32_t* n_pad,
                    const int32_t* k_pad, const int32_t* n_real, float* logits, int32_t n_classes,
                    int32_t* error_flag, void* stream);

/* dz = dy * GELU'(z) elementwise (BF16 and/or FP32 outputs). */
int pb_mlp_gelu_backward(const float* dy, const float* z, int64_t n, void* dz_bf16, float* dz_f32, void* stream);
/* Softmax cross-entropy of (M x C) logits against labels (NULL: no loss):
 * dz = (softmax - onehot) * scale; loss_sum += sum of -log p[label];
 * correct += number of rows whose argmax is the label. */
int pb_mlp_softmax_xent(const float* logits, const int32_t* labels, int32_t M, int32_t C, float scale,
                        void* dz_bf16, float* dz_f32, float* loss_sum, int32_t* correct, void* stream);
/* db[n] = alpha * sum_m dz[m, n] for an (M x N) FP32 matrix. */
int pb_mlp_bias_grad(const float* dz, int32_t M, int32_t N, float alpha, float* db, void* stream);
/* AdamW step `step` (>= 1) on FP32 master weights; refreshes the BF16 copy if given. */
int pb_mlp_adamw(float* w, const float* g, float* m1, float* m2, void* w_bf16, int64_t n, float lr,
                 float beta1, float beta2, float eps, float weight_decay, int32_t step, void* stream);
/* y = BF16(x). */
int pb_mlp_cast_bf16(const float* x, void* y, int64_t n, void* stream);
/* Network inputs, as BF16 rows zero padded to d_pad columns: z = [(ic[r, :S],
 * params[:n_params]) - shift] * scale (d = S + n_params columns), then, for the
 * n_freq rows f of freq (n_freq x d, cycles per unit of z), sin(2 pi f.z) for
 * every f and cos(2 pi f.z) for every f (random Fourier features; n_freq = 0
 * and freq = NULL for z alone).  d = S + n_params <= 16, n_freq <= 128,
 * d + 2 n_freq <= d_pad. */
int pb_surrogate_inputs(const float* ic, int32_t S, const double* params, int32_t n_params, const float* shift,
                        const float* scale, const float* freq, int32_t n_freq, int64_t n, int32_t d_pad,
                        void* out_bf16, void* stream);
/* The same with a parameter row per IC (parameter studies): params is an
 * (n_param_rows x n_params) FP64 table and row r of the inputs takes row
 * param_index[r] (NULL: row 0); an index outside the table gives NaN inputs,
 * which the gate routes to the integrator. */
int pb_surrogate_inputs_rows(const float* ic, int32_t S, const double* params, int64_t n_param_rows,
                             int32_t n_params, const int32_t* param_index, const float* shift, const float* scale,
                             const float* freq, int32_t n_freq, int64_t n, int32_t d_pad, void* out_bf16,
                             void* stream);
/* Confidence gate: label = argmax, conf = max softmax probability; rows with
 * conf < threshold (or not finite) or audit[i] != 0 are appended to route
 * (n_route counts them, reset by the call). */
int pb_surrogate_gate(const float* logits, int64_t n, int32_t C, float threshold, const uint8_t* audit,
                      int32_t* label, float* conf, int32_t* route, int32_t* n_route, void* stream);
/* y[k, :] = x[idx[k], :] for k < min(*n_idx, max_rows). */
int pb_gather_rows(const float* x, int32_t width, const int32_t* idx, const int32_t* n_idx, int64_t max_rows,
                   float* y, void* stream);
/* label[idx[k]] = integrated[k] for k < min(*n_idx, max_rows); the surrogate's label of
 * each routed row is kept in surrogate_label_of_routed[k] (may be NULL). */
int pb_merge_labels(const int32_t* integrated, const int32_t* idx, const int32_t* n_idx, int64_t max_rows,
                    int32_t* label, int32_t* surrogate_label_of_routed, void* stream);
/* Summary of a gated pass, without host round trips: counts[c] (int64, C <= 64)
 * of the final labels, and over the routed rows (route[:min(*n_route, max_rows)];
 * route may be NULL for none) the audit tally stats[0] = audited rows, stats[1] =
 * those whose surrogate confidence conf[i] was >= threshold, stats[2] = those of
 * them whose surrogate label (surrogate_label_of_routed[q]) differs from the
 * integrator's (integrated[q]).  counts and stats are cleared by the call.  No
 * counterpart in the reference (the surrogate gate is this library's own). */
int pb_gate_summary(const int32_t* label, int64_t n, int32_t C, const int32_t* route, const int32_t* n_route,
                    int64_t max_rows, const uint8_t* audit, const float* conf, float threshold,
                    const int32_t* surrogate_label_of_routed, const int32_t* integrated, int64_t* counts,
                    int32_t* stats, void* stream);

/* ---- surrogate training on the tensor cores (tcgen05) ----------------------
 * No counterpart in the reference.  One minibatch step of the surrogate is
 * forward GEMMs (PB_TRAIN_FWD_GELU, PB_TRAIN_FWD_LINEAR for the logits),
 * pb_train_xent, input-gradient GEMMs (PB_TRAIN_DX) and weight-gradient GEMMs
 * (PB_TRAIN_DW), then pb_train_adamw; nothing allocates, so a whole training
 * run can be captured as one CUDA graph. */
enum pb_train_mode {
    PB_TRAIN_FWD_GELU = 0,   /* out_bf16 = GELU(A B^T + bias) (BF16), z_pre = A B^T + bias (FP32, optional) */
    PB_TRAIN_FWD_LINEAR = 1, /* out_f32 = A B^T + bias (bias optional) */
    PB_TRAIN_DX = 2,         /* out_bf16 = (A B^T) * GELU'(z_in); col_part (optional) per-warp column sums */
    PB_TRAIN_DW = 3          /* out_f32 + z * M * ldc = A B^T over K chunk z (split-K partials); with
                                col_part, col_part[z * ldp + m] = sum over the chunk of A(m, k) (the bias
                                gradient partial: B gets a virtual row N of ones) */
};
/* C (M x N) = A (M x K) B^T with B given as (N x K): A(m,k) = A[m*sam + k*sak],
 * B(n,k) = B[n*sbn + k*sbk] (BF16, device); each operand is contiguous along K
 * (sak = 1 / sbk = 1) or along its rows (sam = 1 / sbn = 1; slower: staged by
 * scattered shared-memory stores).  out_t (optional, BF16 modes) receives the BF16
 * output transposed, out_t[n * ldt + m], so that a following weight-gradient GEMM
 * reads it contiguous along K.  A CTA computes 128
 * rows x bn columns over a K chunk of kc (bn, kc multiples of 16, <= 256) with
 * tcgen05.mma, FP32 accumulators in tensor memory; the forward and input-gradient
 * modes need kc >= K.  Outputs have row stride ldc; col_part has row stride ldp
 * and ceil(M / 128) * 4 rows for PB_TRAIN_DX, ceil(K / kc) rows for PB_TRAIN_DW.
 * error_flag (device int32, optional) is set to 1 when a CTA gave up waiting
 * for its MMAs. */
int pb_train_gemm(const void* A, int64_t sam, int64_t sak, const void* B, int64_t sbn, int64_t sbk, int32_t M,
                  int32_t N, int32_t K, int32_t mode, int32_t kc, int32_t bn, const float* bias, const float* z_in,
                  int64_t ldz, float* out_f32, void* out_bf16, void* out_t, float* z_pre, float* col_part,
                  int64_t ldc, int64_t ldt, int64_t ldp, int32_t* error_flag, void* stream);
/* Softmax cross-entropy of logits (M x C, row stride ldl; C <= 32) against
 * labels: dz = (softmax - onehot) * scale (BF16, row stride ldd; dz_t, optional,
 * the same transposed: dz_t[c * ldt + m]); bias_part
 * (optional) receives pb_train_xent_parts(M) rows of C column sums of dz;
 * loss_sum and correct (optional) accumulate -log p[label] and argmax hits. */
int pb_train_xent(const float* logits, int64_t ldl, const int32_t* labels, int32_t M, int32_t C, float scale,
                  void* dz_bf16, int64_t ldd, void* dz_t, int64_t ldt, float* bias_part, float* loss_sum,
                  int32_t* correct, void* stream);
int pb_train_xent_parts(int32_t M);
/* AdamW step `step` (>= 1) over n_tensors (<= 16) parameter tensors in one
 * launch.  Tensor s: FP32 weights w[s] (n[s] = rows x cols[s], row-major),
 * optional BF16 copy w_bf16[s] and transposed BF16 copy w_bf16_t[s] (cols x
 * rows; w_bf16, w_bf16_t and cols may be NULL), moments m1[s], m2[s], and its
 * gradient as n_parts[s] partials summed in order, partial p of element i at
 * grad_parts[s][p * part_stride[s] + i]; weight_decay[s] per tensor.  The
 * pointer arrays are host arrays. */
int pb_train_adamw(int32_t n_tensors, float* const* w, void* const* w_bf16, void* const* w_bf16_t,
                   const int64_t* cols, float* const* m1, float* const* m2, const float* const* grad_parts,
                   const int64_t* n, const int64_t* part_stride, const int32_t* n_parts, const float* weight_decay,
                   float lr, float beta1, float beta2, float eps, int32_t step, void* stream);
/* out[k, :] = x[idx[k], :] (BF16 rows of `width`), out_t[c * n + k] = the same
 * transposed (optional), labels_out[k] = labels[idx[k]] (optional), k < n: the
 * shuffled copy of a training set for one epoch. */
int pb_train_gather(const void* x_bf16, int32_t width, const int32_t* labels, const int32_t* idx, int64_t n,
                    void* out_bf16, void* out_t, int32_t* labels_out, void* stream);

/* ---- fused training step (tcgen05) ------------------------------------------
 * No counterpart in the reference.  One minibatch step of an MLP with layer
 * widths dims[0..n_layers] (GELU between layers, softmax cross-entropy on the
 * dims[n_layers] logits, AdamW) as two launches: one CTA per 128 rows runs the
 * forward pass, the loss and the input gradients of its rows; one cluster per
 * weight tile sums the weight gradient over the minibatch and applies AdamW.
 * Limits: 1 <= n_layers <= PB_TRAIN_MAX_LAYERS, dims[0] a multiple of 8 in
 * [8, 256], hidden widths multiples of 16 in [16, 256], 2 <= dims[n_layers] <= 32.
 *
 * Parameters live augmented: layer l is an FP32 (npad_l x kaug_l) row-major
 * matrix [W_l | b_l | 0] (npad_l = dims[l+1] rounded up to 16 with zero rows,
 * kaug_l = dims[l] + 1 rounded up to 16; the bias in column dims[l]), all layers
 * concatenated at element offsets aug_off_l; AdamW moments m1, m2 have the same
 * shape; w_img holds the BF16 weight images the kernels read (img_bytes). */
#define PB_TRAIN_MAX_LAYERS 8
/* Sizes for a network and minibatch size `batch`: out[0] = img_bytes, out[1] =
 * scratch bytes, out[2] = augmented elements; then per layer l: out[3+4l] =
 * kaug_l, out[4+4l] = npad_l, out[5+4l] = aug_off_l, out[6+4l] = byte offset
 * of the layer's image.  out_len >= 3 + 4 n_layers. */
int pb_train_fused_geometry(int32_t n_layers, const int32_t* dims, int32_t batch, int64_t* out, int32_t out_len);
/* w_img = the BF16 images of the augmented weights w_aug (device). */
int pb_train_fused_pack(int32_t n_layers, const int32_t* dims, const float* w_aug, void* w_img, void* stream);
/* One minibatch step over rows[0..M) (M <= batch) of the training set x (BF16,
 * n_rows x dims[0], 16-byte aligned) with int32 labels; a row index outside
 * [0, n_rows) is not read (the row counts as zero and error_flag is set).  grad NULL: AdamW step `step`
 * (>= 1; weight decay on the weights, not the bias) on w_aug, m1, m2, w_img.
 * grad non-NULL: the minibatch-mean gradient (augmented layout) is written to
 * grad and nothing is updated.  loss_sum / correct (optional) accumulate the
 * summed loss and argmax hits; error_flag (optional) is set to 1 when a wait gave
 * up.  scratch: the geometry's scratch bytes for `batch`, 16-byte aligned. */
int pb_train_fused_step(int32_t n_layers, const int32_t* dims, const void* x_bf16, const int32_t* labels,
                        int32_t n_rows, const int32_t* rows, int32_t M, int32_t batch, float* w_aug, float* m1, float* m2,
                        void* w_img, void* scratch, float* grad, float lr, float beta1, float beta2, float eps,
                        float weight_decay, int32_t step, float* loss_sum, int32_t* correct, int32_t* error_flag,
                        void* stream);
/* Inference with the same BF16 weight images: logits (n x dims[n_layers], FP32) of
 * the BF16 inputs x (n x dims[0], 16-byte aligned).  Persistent CTAs take pairs of
 * 128-row tiles and alternate between them, so one tile's MMAs run while the other
 * tile's activations are computed.  error_flag (optional) as for the step. */
int pb_mlp_infer_fused(int32_t n_layers, const int32_t* dims, const void* x_bf16, int64_t n, const void* w_img,
                       float* logits, int32_t* error_flag, void* stream);
/* AdamW step from a gradient in the augmented layout (e.g. after a data-parallel
 * all-reduce of pb_train_fused_step's grad output), refreshing w_img. */
int pb_train_fused_adamw(int32_t n_layers, const int32_t* dims, float* w_aug, float* m1, float* m2, const float* grad,
                         void* w_img, float lr, float beta1, float beta2, float eps, float weight_decay, int32_t step,
                         void* stream);

/* Human-readable text of a pb_status (src/zigode/zig_solver.py:333-341). */
const char* pb_error_string(int32_t status);

/* ABI version (major*100 + minor). */
int32_t pb_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PYBASIN_B200_H */
