/* FP64 CPU oracle: test infrastructure only (see dopri5_oracle.c). */
#ifndef PB_ORACLE_H
#define PB_ORACLE_H
#include <stdint.h>

enum {
    ORACLE_SYS_LINEAR = 0,
    ORACLE_SYS_PENDULUM = 1,
    ORACLE_SYS_DUFFING = 2,
    ORACLE_SYS_LORENZ = 3,
    ORACLE_SYS_LORENZ_MASKED = 4,
    ORACLE_SYS_ROSSLER_NET = 5,
    ORACLE_SYS_FRICTION = 6,
};

/* feature kinds: same numbering as the CUDA library's PB_FEAT_* */
enum {
    ORACLE_F_MEDIAN = 0, ORACLE_F_MEAN = 1, ORACLE_F_STD = 2, ORACLE_F_VAR = 3, ORACLE_F_RMS = 4,
    ORACLE_F_MAX = 5, ORACLE_F_ABSMAX = 6, ORACLE_F_MIN = 7, ORACLE_F_DELTA = 8,
    ORACLE_F_LOG_DELTA = 9, ORACLE_F_AMPLITUDE = 10, ORACLE_F_CROSSINGS = 11, ORACLE_F_LAST = 12,
    /* 13 is the network-only synchronisation feature */
    ORACLE_F_SUM = 14, ORACLE_F_ABS_ENERGY = 15, ORACLE_F_LENGTH = 16, ORACLE_F_VARIATION_COEFF = 17,
    ORACLE_F_QUANTILE = 18, ORACLE_F_KURTOSIS = 19, ORACLE_F_SKEWNESS = 20, ORACLE_F_ABS_SUM_CHANGES = 21,
    ORACLE_F_MEAN_ABS_CHANGE = 22, ORACLE_F_MEAN_CHANGE = 23, ORACLE_F_MEAN_SECOND_DERIV = 24,
    ORACLE_F_COUNT_ABOVE_MEAN = 25, ORACLE_F_COUNT_BELOW_MEAN = 26, ORACLE_F_COUNT_ABOVE = 27,
    ORACLE_F_COUNT_BELOW = 28, ORACLE_F_NUMBER_PEAKS = 29, ORACLE_F_AUTOCORRELATION = 30,
    ORACLE_F_RATIO_BEYOND_R_SIGMA = 31,
    /* fft_coefficient real/imag/abs/angle (coeff), linear_trend slope/intercept/
       rvalue/pvalue/stderr, first/last location of max/min, cid_ce (normalize),
       c3 (lag), time_reversal_asymmetry_statistic (lag) */
    ORACLE_F_FFT_REAL = 32, ORACLE_F_FFT_IMAG = 33, ORACLE_F_FFT_ABS = 34, ORACLE_F_FFT_ANGLE = 35,
    ORACLE_F_TREND_SLOPE = 36, ORACLE_F_TREND_INTERCEPT = 37, ORACLE_F_TREND_RVALUE = 38,
    ORACLE_F_TREND_PVALUE = 39, ORACLE_F_TREND_STDERR = 40,
    ORACLE_F_FIRST_LOC_MAX = 41, ORACLE_F_FIRST_LOC_MIN = 42, ORACLE_F_LAST_LOC_MAX = 43,
    ORACLE_F_LAST_LOC_MIN = 44, ORACLE_F_CID_CE = 45, ORACLE_F_C3 = 46, ORACLE_F_TIME_REVERSAL = 47,
    /* spkt_welch_density (coeff), large_standard_deviation (r), symmetry_looking (r),
       index_mass_quantile (q), longest_strike_above_mean, longest_strike_below_mean */
    ORACLE_F_SPKT_WELCH = 48, ORACLE_F_LARGE_STD = 49, ORACLE_F_SYMMETRY_LOOKING = 50,
    ORACLE_F_INDEX_MASS_QUANTILE = 51, ORACLE_F_LONGEST_STRIKE_ABOVE = 52, ORACLE_F_LONGEST_STRIKE_BELOW = 53,
    /* has_duplicate_max, has_duplicate_min, binned_entropy (max_bins),
       mean_n_absolute_max (number_of_maxima), benford_correlation */
    ORACLE_F_HAS_DUP_MAX = 54, ORACLE_F_HAS_DUP_MIN = 55, ORACLE_F_BINNED_ENTROPY = 56,
    ORACLE_F_MEAN_N_ABS_MAX = 57, ORACLE_F_BENFORD = 58,
    /* has_duplicate, percentage_of_reoccurring_datapoints_to_all_datapoints,
       percentage_of_reoccurring_values_to_all_values, sum_of_reoccurring_data_points,
       sum_of_reoccurring_values, ratio_value_number_to_time_series_length,
       has_variance_larger_than_standard_deviation, count_value (value) */
    ORACLE_F_HAS_DUPLICATE = 59, ORACLE_F_PCT_REOCCURRING_POINTS = 60, ORACLE_F_PCT_REOCCURRING_VALUES = 61,
    ORACLE_F_SUM_REOCCURRING_POINTS = 62, ORACLE_F_SUM_REOCCURRING_VALUES = 63, ORACLE_F_RATIO_UNIQUE_VALUES = 64,
    ORACLE_F_VAR_LARGER_THAN_STD = 65, ORACLE_F_COUNT_VALUE = 66,
    /* partial_autocorrelation (lag), agg_autocorrelation (maxlag; mean, median, var),
       energy_ratio_by_chunks (num_segments, segment_focus), count_in_range (min_val,
       max_val), change_quantiles (ql, qh; isabs x f_agg mean / var) */
    ORACLE_F_PARTIAL_AUTOCORRELATION = 67, ORACLE_F_AGG_AUTOCORR_MEAN = 68, ORACLE_F_AGG_AUTOCORR_MEDIAN = 69,
    ORACLE_F_AGG_AUTOCORR_VAR = 70, ORACLE_F_ENERGY_RATIO_BY_CHUNKS = 71, ORACLE_F_COUNT_IN_RANGE = 72,
    ORACLE_F_CHANGE_QUANTILES_MEAN = 73, ORACLE_F_CHANGE_QUANTILES_VAR = 74,
    ORACLE_F_CHANGE_QUANTILES_ABS_MEAN = 75, ORACLE_F_CHANGE_QUANTILES_ABS_VAR = 76,
    /* autocorrelation_periodicity (min_lag, peak_threshold; output strength / period) */
    ORACLE_F_ACF_PERIOD_STRENGTH = 77, ORACLE_F_ACF_PERIOD_LAG = 78,
    /* spectral_frequency_ratio, fft_aggregated (centroid, variance, skew, kurtosis) */
    ORACLE_F_SPECTRAL_FREQ_RATIO = 79, ORACLE_F_FFT_AGG_CENTROID = 80, ORACLE_F_FFT_AGG_VARIANCE = 81,
    ORACLE_F_FFT_AGG_SKEW = 82, ORACLE_F_FFT_AGG_KURTOSIS = 83,
    /* fourier_entropy (bins, unused by the reference), permutation_entropy (tau,
       dimension), lempel_ziv_complexity (bins) */
    ORACLE_F_FOURIER_ENTROPY = 84, ORACLE_F_PERMUTATION_ENTROPY = 85, ORACLE_F_LEMPEL_ZIV = 86,
    /* agg_linear_trend (chunk_size, attr index 0..4 = slope, intercept, rvalue,
       pvalue, stderr; f_agg mean / var / min / max), ar_coefficient (k <= 10, coeff) */
    ORACLE_F_AGG_TREND_MEAN = 87, ORACLE_F_AGG_TREND_VAR = 88, ORACLE_F_AGG_TREND_MIN = 89,
    ORACLE_F_AGG_TREND_MAX = 90, ORACLE_F_AR_COEFFICIENT = 91,
    /* cwt_coefficients (w, coeff; coeff < 0: w not among the widths -> 0),
       friedrich_coefficients (m <= 6, coeff), max_langevin_fixed_point (m <= 6) */
    ORACLE_F_CWT = 92, ORACLE_F_FRIEDRICH = 93, ORACLE_F_LANGEVIN = 94,
    /* augmented_dickey_fuller (teststat, pvalue, usedlag), number_cwt_peaks (max_width) */
    ORACLE_F_ADF_TESTSTAT = 95, ORACLE_F_ADF_PVALUE = 96, ORACLE_F_ADF_USEDLAG = 97, ORACLE_F_NUMBER_CWT_PEAKS = 98,
    /* correlation_dimension (emb_dim; param2 = lag * 1024 + n_rvals) */
    ORACLE_F_CORR_DIM = 99,
    /* lyapunov_r (param = emb_dim * 1024 + trajectory_len, param2 = lag; tau = 1) */
    ORACLE_F_LYAP_R = 100,
};
#define ORACLE_MAX_ACF_LAG 63 /* partial_autocorrelation lags held on the stack */

enum { ORACLE_OK = 0, ORACLE_MAX_STEPS = 1, ORACLE_DT_UNDERFLOW = 2, ORACLE_UNBOUNDED = 3, ORACLE_NONFINITE = 4 };
enum { ORACLE_EINVAL = -5, ORACLE_ENOMEM = -2 };

typedef struct {
    const int32_t *row_ptr; /* CSR adjacency for network systems (n_nodes + 1) */
    const int32_t *col_idx;
} oracle_aux;

typedef struct {
    int32_t system;
    int32_t dim;
    int32_t n_params;
    int32_t n_save;
    int32_t win_begin;      /* first save index inside the feature window */
    int32_t n_features;
    double t0, t1;
    const double *save_ts;  /* (n_save,) */
    double rtol, atol;
    int64_t max_steps;
    double unbounded_thr;   /* <= 0: off */
    const int32_t *feat_state; /* (n_features,) */
    const int32_t *feat_kind;  /* (n_features,) */
    const double *feat_param;  /* (n_features,) or NULL */
    const oracle_aux *aux;
    const double *feat_param2; /* (n_features,) second parameter of the two-parameter kinds, or NULL */
} oracle_problem;

int oracle_solve_batch(const oracle_problem *pb, const double *y0s, int64_t n_traj,
                       const double *params, const int32_t *param_index, double *features_out,
                       int32_t *status_out, double *y_final, double *y_full, int64_t *steps_out,
                       int64_t *accepted_out, int n_threads);
double oracle_window_feature(int kind, double param, const double *w, int n);
double oracle_window_feature2(int kind, double param, double param2, const double *w, int n);
#endif
