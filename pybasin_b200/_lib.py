"""ctypes binding of the C ABI declared in ``include/pybasin_b200.h``.

The library is built in-tree (``pybasin_b200/_lib/libpybasin_b200.so``).  There
is no CPU fallback: if the library is missing or CUDA is unavailable, every
compute entry point raises.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

from pybasin_b200 import build as _build

# ---- enums mirrored from include/pybasin_b200.h ---------------------------
PB_SUCCESS = 0
PB_EINVALID_ODE = -1
PB_EALLOC = -2
PB_ESOLVE = -3
PB_EINVAL = -5
PB_ECUDA = -6
PB_EUNSUPPORTED = -7
PB_ECOMPILE = -8
PB_ESCRATCH_LIMIT = -9
NOALLOC_SCRATCH_BYTES = 64 * 1024 * 1024

SYS_LINEAR = 0
SYS_PENDULUM = 1
SYS_DUFFING = 2
SYS_LORENZ = 3
SYS_LORENZ_MASKED = 4
SYS_ROSSLER_NET = 5
SYS_FRICTION = 6
SYS_USER = 64

PREC_FP64 = 0
PREC_MIXED = 1

LAYOUT_SINGLE = 0
LAYOUT_CROSS = 1
LAYOUT_INDEXED = 2

SCHED_PLAIN = 0
SCHED_QUEUE = 1
SCHED_PROBED = 2
SCHEDULES = {"plain": SCHED_PLAIN, "queue": SCHED_QUEUE, "probed": SCHED_PROBED}

DENSE_INLINE = 0
DENSE_DEFERRED = 1

DTYPE_F32 = 0
DTYPE_F64 = 1

FEAT_MEDIAN = 0
FEAT_MEAN = 1
FEAT_STD = 2
FEAT_VAR = 3
FEAT_RMS = 4
FEAT_MAX = 5
FEAT_ABSMAX = 6
FEAT_MIN = 7
FEAT_DELTA = 8
FEAT_LOG_DELTA = 9
FEAT_AMPLITUDE = 10
FEAT_CROSSINGS = 11
FEAT_LAST = 12
FEAT_SYNC_DEV = 13
FEAT_SUM = 14
FEAT_ABS_ENERGY = 15
FEAT_LENGTH = 16
FEAT_VARIATION_COEFF = 17
FEAT_QUANTILE = 18
FEAT_KURTOSIS = 19
FEAT_SKEWNESS = 20
FEAT_ABS_SUM_CHANGES = 21
FEAT_MEAN_ABS_CHANGE = 22
FEAT_MEAN_CHANGE = 23
FEAT_MEAN_SECOND_DERIV = 24
FEAT_COUNT_ABOVE_MEAN = 25
FEAT_COUNT_BELOW_MEAN = 26
FEAT_COUNT_ABOVE = 27
FEAT_COUNT_BELOW = 28
FEAT_NUMBER_PEAKS = 29
FEAT_AUTOCORRELATION = 30
FEAT_RATIO_BEYOND_R_SIGMA = 31
FEAT_FFT_REAL, FEAT_FFT_IMAG, FEAT_FFT_ABS, FEAT_FFT_ANGLE = 32, 33, 34, 35
FEAT_TREND_SLOPE, FEAT_TREND_INTERCEPT, FEAT_TREND_RVALUE, FEAT_TREND_PVALUE, FEAT_TREND_STDERR = 36, 37, 38, 39, 40
FEAT_FIRST_LOC_MAX, FEAT_FIRST_LOC_MIN, FEAT_LAST_LOC_MAX, FEAT_LAST_LOC_MIN = 41, 42, 43, 44
FEAT_CID_CE, FEAT_C3, FEAT_TIME_REVERSAL = 45, 46, 47
FEAT_SPKT_WELCH, FEAT_LARGE_STD, FEAT_SYMMETRY_LOOKING = 48, 49, 50
FEAT_INDEX_MASS_QUANTILE, FEAT_LONGEST_STRIKE_ABOVE, FEAT_LONGEST_STRIKE_BELOW = 51, 52, 53
FEAT_HAS_DUP_MAX, FEAT_HAS_DUP_MIN, FEAT_BINNED_ENTROPY, FEAT_MEAN_N_ABS_MAX, FEAT_BENFORD = 54, 55, 56, 57, 58
FEAT_HAS_DUPLICATE, FEAT_PCT_REOCCURRING_POINTS, FEAT_PCT_REOCCURRING_VALUES = 59, 60, 61
FEAT_SUM_REOCCURRING_POINTS, FEAT_SUM_REOCCURRING_VALUES, FEAT_RATIO_UNIQUE_VALUES = 62, 63, 64
FEAT_VAR_LARGER_THAN_STD, FEAT_COUNT_VALUE = 65, 66
FEAT_PARTIAL_AUTOCORRELATION, FEAT_AGG_AUTOCORR_MEAN, FEAT_AGG_AUTOCORR_MEDIAN, FEAT_AGG_AUTOCORR_VAR = 67, 68, 69, 70
FEAT_ENERGY_RATIO_BY_CHUNKS, FEAT_COUNT_IN_RANGE = 71, 72
FEAT_CHANGE_QUANTILES_MEAN, FEAT_CHANGE_QUANTILES_VAR = 73, 74
FEAT_CHANGE_QUANTILES_ABS_MEAN, FEAT_CHANGE_QUANTILES_ABS_VAR = 75, 76
FEAT_ACF_PERIOD_STRENGTH, FEAT_ACF_PERIOD_LAG = 77, 78
FEAT_SPECTRAL_FREQ_RATIO, FEAT_FFT_AGG_CENTROID, FEAT_FFT_AGG_VARIANCE = 79, 80, 81
FEAT_FFT_AGG_SKEW, FEAT_FFT_AGG_KURTOSIS = 82, 83
FEAT_FOURIER_ENTROPY, FEAT_PERMUTATION_ENTROPY, FEAT_LEMPEL_ZIV = 84, 85, 86
FEAT_AGG_TREND_MEAN, FEAT_AGG_TREND_VAR, FEAT_AGG_TREND_MIN, FEAT_AGG_TREND_MAX = 87, 88, 89, 90
FEAT_AR_COEFFICIENT = 91
FEAT_CWT, FEAT_FRIEDRICH, FEAT_LANGEVIN = 92, 93, 94
FEAT_ADF_TESTSTAT, FEAT_ADF_PVALUE, FEAT_ADF_USEDLAG, FEAT_NUMBER_CWT_PEAKS = 95, 96, 97, 98
FEAT_CORR_DIM, FEAT_LYAP_R = 99, 100
SPECTRAL_WINDOW_MAX = 16384  # PB_SPECTRAL_WINDOW_MAX: window samples of the spectral kinds 79..84
SYMBOLIC_WINDOW_MAX = 8191  # PB_SYMBOLIC_WINDOW_MAX: window samples of lempel_ziv_complexity
SORTED_WINDOW_MAX = 32768  # PB_SORTED_WINDOW_MAX: window samples of the sorted kinds 59..64

TRAJ_OK = 0
TRAJ_MAX_STEPS = 1
TRAJ_DT_UNDERFLOW = 2
TRAJ_UNBOUNDED = 3
TRAJ_NONFINITE = 4
TRAJ_BAD_INPUT = 5

MAX_FEATURES = 32
MAX_CROSSING = 4
MAX_PARAMS = 8
MAX_USER_DIM = 16

_c_i32 = ctypes.c_int32
_c_i64 = ctypes.c_int64
_c_dbl = ctypes.c_double
_c_vp = ctypes.c_void_p


class SolveArgs(ctypes.Structure):
    """Mirror of ``pb_solve_args``."""

    _fields_ = [
        ("system", _c_i32),
        ("dim", _c_i32),
        ("precision", _c_i32),
        ("schedule", _c_i32),
        ("layout", _c_i32),
        ("y0_dtype", _c_i32),
        ("n_params", _c_i32),
        ("block_size", _c_i32),
        ("grid_blocks", _c_i32),
        ("_pad0", _c_i32),
        ("n_ic", _c_i64),
        ("n_param_rows", _c_i64),
        ("n_traj", _c_i64),
        ("y0", _c_vp),
        ("params", _c_vp),
        ("param_index", _c_vp),
        ("csr_row", _c_vp),
        ("csr_col", _c_vp),
        ("t0", _c_dbl),
        ("t1", _c_dbl),
        ("save_ts", _c_vp),
        ("n_save", _c_i32),
        ("win_begin", _c_i32),
        ("rtol", _c_dbl),
        ("atol", _c_dbl),
        ("max_steps", _c_i64),
        ("unbounded_thr", _c_dbl),
        ("n_features", _c_i32),
        ("_pad1", _c_i32),
        ("feat_state", _c_i32 * MAX_FEATURES),
        ("feat_kind", _c_i32 * MAX_FEATURES),
        ("feat_param", _c_dbl * MAX_FEATURES),
        ("features_out", _c_vp),
        ("status_out", _c_vp),
        ("y_final_out", _c_vp),
        ("y_full_out", _c_vp),
        ("y_out_dtype", _c_i32),
        ("_pad2", _c_i32),
        ("steps_out", _c_vp),
        ("queue_counter", _c_vp),
        ("scratch", _c_vp),
        ("order", _c_vp),
        ("dense_mode", _c_i32),
        ("window_record_cap", _c_i32),
        ("peaks_out", _c_vp),
        ("peak_cap", _c_i32),
        ("refill_lanes", _c_i32),
        ("feat_param2", _c_dbl * MAX_FEATURES),
    ]


class PbError(RuntimeError):
    """A pb_* entry point returned a non-zero status."""

    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where} failed: {error_string(code)} (code {code})")


_lock = threading.Lock()
_lib: ctypes.CDLL | None = None

EXPORTED_SYMBOLS = (
    "pb_solve_batch",
    "pb_solve_scratch_bytes",
    "pb_label_nearest",
    "pb_query_occupancy",
    "pb_error_string",
    "pb_abi_version",
    "pb_probe_fma",
    "pb_solve_batch_noalloc",
    "pb_morton_keys",
    "pb_morton_order_scratch_bytes",
    "pb_morton_order",
    "pb_rhs_compile",
    "pb_solve_batch_rhs",
    "pb_rhs_release",
)


def library_path() -> Path:
    return _build.lib_path()


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Load (building first if needed) the CUDA library; raises if it cannot."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if build_if_missing and _build.is_stale():
            _build.build()
        if not path.exists():
            raise RuntimeError(
                f"pybasin_b200 CUDA library not found at {path}; build it with `python -m pybasin_b200.build`"
            )
        lib = ctypes.CDLL(str(path))
        lib.pb_solve_batch.restype = ctypes.c_int
        lib.pb_solve_batch.argtypes = [ctypes.POINTER(SolveArgs), _c_vp]
        lib.pb_solve_batch_noalloc.restype = ctypes.c_int
        lib.pb_solve_batch_noalloc.argtypes = [ctypes.POINTER(SolveArgs), _c_vp]
        lib.pb_solve_scratch_bytes.restype = _c_i64
        lib.pb_solve_scratch_bytes.argtypes = [ctypes.POINTER(SolveArgs)]
        lib.pb_label_nearest.restype = ctypes.c_int
        lib.pb_label_nearest.argtypes = [
            _c_vp, _c_i64, _c_i32, _c_vp, _c_i32, _c_vp, _c_i32, _c_vp, _c_vp, _c_i32, _c_vp, _c_vp, _c_vp,
        ]
        lib.pb_rhs_compile.restype = ctypes.c_int
        lib.pb_rhs_compile.argtypes = [
            ctypes.POINTER(ctypes.c_char_p), _c_i32, _c_i32, ctypes.c_char_p, _c_i32,
            ctypes.POINTER(ctypes.c_char_p), _c_i32, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p),
            ctypes.c_char_p, _c_i64,
        ]
        lib.pb_solve_batch_rhs.restype = ctypes.c_int
        lib.pb_solve_batch_rhs.argtypes = [_c_vp, ctypes.POINTER(SolveArgs), _c_vp]
        lib.pb_rhs_release.restype = ctypes.c_int
        lib.pb_rhs_release.argtypes = [_c_vp]
        lib.pb_morton_keys.restype = ctypes.c_int
        lib.pb_morton_keys.argtypes = [_c_vp, _c_i32, _c_i64, _c_i32, _c_i32, _c_vp, _c_vp, _c_vp, _c_vp]
        lib.pb_morton_order_scratch_bytes.restype = _c_i64
        lib.pb_morton_order_scratch_bytes.argtypes = [_c_i64]
        lib.pb_morton_order.restype = ctypes.c_int
        lib.pb_morton_order.argtypes = [_c_vp, _c_i64, _c_i32, _c_vp, _c_i64, _c_vp, _c_vp]
        lib.pb_query_occupancy.restype = ctypes.c_int
        lib.pb_query_occupancy.argtypes = [
            _c_i32, _c_i32, _c_i32, _c_i32, _c_i32, ctypes.POINTER(_c_i32), ctypes.POINTER(_c_i32),
        ]
        lib.pb_error_string.restype = ctypes.c_char_p
        lib.pb_error_string.argtypes = [_c_i32]
        lib.pb_probe_fma.restype = ctypes.c_int
        lib.pb_probe_fma.argtypes = [_c_i32, _c_i32, _c_i32, _c_vp, _c_vp]
        lib.pb_abi_version.restype = _c_i32
        lib.pb_abi_version.argtypes = []
        _lib = lib
        return lib


def error_string(code: int) -> str:
    try:
        return load(build_if_missing=False).pb_error_string(code).decode()
    except Exception:  # library unavailable: still produce a message
        return f"pb status {code}"


def check(code: int, where: str) -> None:
    if code != PB_SUCCESS:
        raise PbError(code, where)
