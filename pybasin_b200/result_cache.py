"""Result cache of B200Dopri5Solver.integrate (the reference's CacheManager,
src/pybasin/cache_manager.py:27-128, with the fused outputs).

Key: MD5 over the solver class, the system's ``get_str`` and sorted parameters, the
bytes of ``y0``, the save grid and the batched parameters, and every solver setting
that changes the result (tolerances, precision, output mode, feature columns and
window start, max steps, unbounded threshold).  Value: a safetensors file with
``t``, ``y``, and in fused mode ``features`` and ``status``.  A corrupt or
unreadable file is treated as a miss and rewritten.
"""

from __future__ import annotations

import hashlib
import logging
import os
import pickle
from typing import Any

import torch
from safetensors.torch import load_file, save_file

logger = logging.getLogger(__name__)


def cache_key(solver: Any, ode_system: Any, y0: torch.Tensor, params: torch.Tensor | None) -> str:
    save = solver.save_times(y0.dtype)
    cols = solver.feature_extractor.columns(y0.shape[1]) if solver.feature_extractor is not None else []
    ts = solver.feature_extractor.resolve_time_steady(save) if cols else None
    config = (
        ("rtol", float(solver.effective_tolerances()[0])),
        ("atol", float(solver.effective_tolerances()[1])),
        ("precision", solver.precision),
        ("output", solver.output),
        ("max_steps", int(solver.max_steps)),
        ("unbounded", float(solver.unbounded_threshold or 0.0)),
        ("columns", tuple((c.state, c.kind, c.param) for c in cols)),
        ("time_steady", ts),
        ("t_span", tuple(float(v) for v in solver.t_span)),
    )
    params_tuple = tuple(sorted(ode_system.params.items())) if hasattr(ode_system, "params") else ()
    get_str = ode_system.get_str() if hasattr(ode_system, "get_str") else type(ode_system).__name__
    data = (
        type(solver).__name__,
        get_str,
        params_tuple,
        y0.detach().cpu().numpy().tobytes(),
        save.detach().cpu().numpy().tobytes(),
        config,
        params.detach().cpu().numpy().tobytes() if params is not None else b"",
    )
    return hashlib.md5(pickle.dumps(data)).hexdigest()


def cached_integrate(solver: Any, ode_system: Any, y0: torch.Tensor, params: torch.Tensor | None):
    from pybasin_b200.solver import IntegrationResult

    key = cache_key(solver, ode_system, y0, params)
    path = os.path.join(solver._cache_dir, f"{key}.safetensors")
    if os.path.exists(path):
        try:
            d = load_file(path, device=str(solver.device))
            y = d["y"]
            feats = d.get("features")
            status = d["status"]
            cols = solver.feature_extractor.columns(y0.shape[1]) if solver.feature_extractor is not None else []
            names = [c.name for c in cols]
            y._pb_features = feats if feats is not None else torch.zeros((y.shape[1], 0), dtype=y0.dtype,
                                                                         device=y.device)
            y._pb_feature_names = names
            y._pb_status = status
            logger.debug("B200Dopri5Solver: result loaded from cache %s", path)
            return IntegrationResult(d["t"], y, features=y._pb_features, feature_names=names, status=status,
                                     steps=None, peaks=None)
        except Exception as exc:  # unreadable file: recompute and overwrite
            logger.warning("B200Dopri5Solver: ignoring unreadable cache file %s (%s)", path, exc)
    res = solver._integrate(ode_system, y0, params, solver.feature_extractor, 0)
    t, y = res
    os.makedirs(solver._cache_dir, exist_ok=True)
    tensors = {"t": t.contiguous(), "y": y.contiguous(), "status": res.status.contiguous()}
    if res.features is not None:
        tensors["features"] = res.features.contiguous()
    tmp = path + f".tmp{os.getpid()}"
    save_file({k: v.detach() for k, v in tensors.items()}, tmp)
    os.replace(tmp, path)
    return res
