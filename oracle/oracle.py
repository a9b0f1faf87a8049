"""ctypes binding of the FP64 CPU oracle (``dopri5_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline / reference arm of ``bench.py`` as the checker.  The product
library never imports this module.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "liboracle.so"

SYS_LINEAR = 0
SYS_PENDULUM = 1
SYS_DUFFING = 2
SYS_LORENZ = 3
SYS_LORENZ_MASKED = 4
SYS_ROSSLER_NET = 5
SYS_FRICTION = 6

STATUS_OK = 0
STATUS_MAX_STEPS = 1
STATUS_DT_UNDERFLOW = 2
STATUS_UNBOUNDED = 3
STATUS_NONFINITE = 4


class _Aux(ctypes.Structure):
    _fields_ = [("row_ptr", ctypes.POINTER(ctypes.c_int32)), ("col_idx", ctypes.POINTER(ctypes.c_int32))]


class _Problem(ctypes.Structure):
    _fields_ = [
        ("system", ctypes.c_int32),
        ("dim", ctypes.c_int32),
        ("n_params", ctypes.c_int32),
        ("n_save", ctypes.c_int32),
        ("win_begin", ctypes.c_int32),
        ("n_features", ctypes.c_int32),
        ("t0", ctypes.c_double),
        ("t1", ctypes.c_double),
        ("save_ts", ctypes.POINTER(ctypes.c_double)),
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("max_steps", ctypes.c_int64),
        ("unbounded_thr", ctypes.c_double),
        ("feat_state", ctypes.POINTER(ctypes.c_int32)),
        ("feat_kind", ctypes.POINTER(ctypes.c_int32)),
        ("feat_param", ctypes.POINTER(ctypes.c_double)),
        ("aux", ctypes.POINTER(_Aux)),
        ("feat_param2", ctypes.POINTER(ctypes.c_double)),
    ]


def build() -> Path:
    """Compile the oracle with its Makefile (gcc + OpenMP) if it is missing or stale."""
    src = _HERE / "dopri5_oracle.c"
    if not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < max(
        src.stat().st_mtime, (_HERE / "oracle.h").stat().st_mtime
    ):
        subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


_lib: ctypes.CDLL | None = None


def _load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(_LIB_PATH))
        lib.oracle_window_feature.restype = ctypes.c_double
        lib.oracle_window_feature.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int]
        lib.oracle_window_feature2.restype = ctypes.c_double
        lib.oracle_window_feature2.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                               ctypes.c_int]
        lib.oracle_solve_batch.restype = ctypes.c_int
        lib.oracle_solve_batch.argtypes = [
            ctypes.POINTER(_Problem),
            ctypes.c_void_p,
            ctypes.c_int64,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_int,
        ]
        _lib = lib
    return _lib


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


def solve_batch(
    system: int,
    y0: np.ndarray,
    params: np.ndarray,
    save_ts: np.ndarray,
    t_span: tuple[float, float],
    rtol: float,
    atol: float,
    *,
    param_index: np.ndarray | None = None,
    win_begin: int = 0,
    features: list[tuple[int, int, float]] | None = None,
    max_steps: int = 1_000_000,
    unbounded_thr: float = 0.0,
    keep_full: bool = False,
    n_threads: int = 0,
    csr: tuple[np.ndarray, np.ndarray] | None = None,
) -> dict[str, np.ndarray]:
    """Integrate every row of ``y0`` with the FP64 oracle.

    :param system: one of the ``SYS_*`` ids.
    :param y0: ``(n_traj, dim)`` initial conditions.
    :param params: ``(n_rows, n_params)`` parameter table.
    :param param_index: ``(n_traj,)`` row of ``params`` per trajectory (default row 0).
    :param features: output columns ``(state, kind, param)`` or ``(state, kind, param,
        param2)`` in output order.
    :return: dict with ``features (n,F)``, ``status (n,)``, ``y_final (n,dim)``,
        ``steps``/``accepted`` ``(n,)`` and, with ``keep_full``, ``y (n_save,n,dim)``.
    """
    lib = _load()
    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    n, dim = y0.shape
    params = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
    save_ts = np.ascontiguousarray(save_ts, dtype=np.float64)
    feats = features or []
    fs = np.ascontiguousarray([f[0] for f in feats] or [0], dtype=np.int32)
    fk = np.ascontiguousarray([f[1] for f in feats] or [0], dtype=np.int32)
    fp = np.ascontiguousarray([f[2] for f in feats] or [0.0], dtype=np.float64)
    fp2 = np.ascontiguousarray([f[3] if len(f) > 3 else 0.0 for f in feats] or [0.0], dtype=np.float64)
    pidx = None if param_index is None else np.ascontiguousarray(param_index, dtype=np.int32)
    aux = None
    keep: list[object] = []
    if csr is not None:
        rp = np.ascontiguousarray(csr[0], dtype=np.int32)
        ci = np.ascontiguousarray(csr[1], dtype=np.int32)
        keep += [rp, ci]
        aux = _Aux(rp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ci.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    pb = _Problem(
        system,
        dim,
        params.shape[1],
        save_ts.shape[0],
        win_begin,
        len(feats),
        float(t_span[0]),
        float(t_span[1]),
        save_ts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        rtol,
        atol,
        max_steps,
        unbounded_thr,
        fs.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
        fk.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
        fp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        ctypes.pointer(aux) if aux is not None else None,
        fp2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
    )
    out_f = np.empty((n, max(len(feats), 1)), dtype=np.float64)
    status = np.empty(n, dtype=np.int32)
    y_final = np.empty((n, dim), dtype=np.float64)
    steps = np.empty(n, dtype=np.int64)
    acc = np.empty(n, dtype=np.int64)
    y_full = np.empty((save_ts.shape[0], n, dim), dtype=np.float64) if keep_full else None
    rc = lib.oracle_solve_batch(
        ctypes.byref(pb),
        _ptr(y0),
        n,
        _ptr(params),
        _ptr(pidx),
        _ptr(out_f) if feats else None,
        _ptr(status),
        _ptr(y_final),
        _ptr(y_full),
        _ptr(steps),
        _ptr(acc),
        n_threads if n_threads > 0 else (os.cpu_count() or 1),
    )
    if rc != 0:
        raise RuntimeError(f"oracle_solve_batch failed with code {rc}")
    res = {"features": out_f[:, : len(feats)], "status": status, "y_final": y_final, "steps": steps, "accepted": acc}
    if y_full is not None:
        res["y"] = y_full
    return res


def window_feature(kind: int, param: float, w: np.ndarray, param2: float = 0.0) -> float:
    """Feature ``kind`` of one stored window ``w`` (two-pass, as the reference's
    calculators); ``param2`` is the second parameter of the two-parameter kinds."""
    lib = _load()
    w = np.ascontiguousarray(w, dtype=np.float64)
    return float(lib.oracle_window_feature2(kind, param, param2, w.ctypes.data, w.shape[0]))


def peak_values(w: np.ndarray, n: int) -> np.ndarray:
    """Values of the strict local maxima of window ``w`` with support ``n`` on each
    side, in time order (find_peak_mask / extract_peak_values,
    src/pybasin/ts_torch/calculators/torch_features_pattern.py:64-150)."""
    w = np.asarray(w, dtype=np.float64)
    out = []
    for i in range(n, len(w) - n):
        if all(w[i] > w[i - j] and w[i] > w[i + j] for j in range(1, n + 1)):
            out.append(w[i])
    return np.array(out)
