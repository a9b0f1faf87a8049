"""The allocation-free entry point, pb_solve_batch_noalloc, through the C ABI.

pb_solve_batch_noalloc serves callers that may not allocate device memory on
demand (a plug-in inside a host application that owns all device memory under a
fixed budget, or a latency-critical loop that cannot afford cudaMalloc): it runs
the same kernels as pb_solve_batch with the integrator's scratch in a fixed
array the library reserves on each GPU.  These tests check that two calls in a
row give the outputs of the allocating entry point on the same inputs, and that
a request too large for the fixed array is refused without a launch.  The file
is named so that pytest collects it last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from pybasin_b200 import _lib as L
from pybasin_b200.engine import FeatureColumn, SolveRequest, SolveResult, alloc_scratch, build_args

pytestmark = pytest.mark.gpu


def _request(dev: torch.device, n: int, schedule: int = L.SCHED_QUEUE) -> SolveRequest:
    torch.manual_seed(5)
    y0 = (torch.rand(n, 2) * torch.tensor([2.0, 1.5]) + torch.tensor([-1.0, -0.5])).to(dev)
    save = torch.linspace(900.0, 1000.0, 5000, dtype=torch.float32).double().to(dev)
    cols = [
        FeatureColumn(0, L.FEAT_MAX),
        FeatureColumn(0, L.FEAT_STD),
        FeatureColumn(0, L.FEAT_MEDIAN),
        FeatureColumn(1, L.FEAT_CROSSINGS, 0.0),
        FeatureColumn(1, L.FEAT_MEAN),
    ]
    return SolveRequest(
        system=L.SYS_DUFFING,
        dim=2,
        y0=y0,
        params=torch.tensor([[0.08, 1.0, 0.2]], dtype=torch.float64, device=dev),
        save_ts=save,
        t_span=(0.0, 1000.0),
        rtol=1e-6,
        atol=1e-6,
        n_traj=n,
        columns=cols,
        precision=L.PREC_MIXED,
        schedule=schedule,
        dense_mode=L.DENSE_DEFERRED,
        keep_steps=True,
    )


def _outputs(req: SolveRequest, dev: torch.device) -> SolveResult:
    n = req.n_traj
    return SolveResult(
        features=torch.full((n, len(req.columns)), float("nan"), dtype=torch.float64, device=dev),
        status=torch.full((n,), -1, dtype=torch.int32, device=dev),
        y_final=torch.zeros((n, req.dim), dtype=torch.float32, device=dev),
        y_full=None,
        steps=torch.zeros((n,), dtype=torch.int64, device=dev),
    )


# the queue schedule, and the probed one (probe phase, longest-first radix sort
# whose temporary storage also lives in the fixed array, main phase with the
# sampling drained into it)
@pytest.mark.parametrize("schedule", [L.SCHED_QUEUE, L.SCHED_PROBED], ids=["queue", "probed"])
def test_noalloc_matches_allocating_entry_point_on_two_calls(schedule):
    dev = torch.device("cuda:0")
    lib = L.load()
    req = _request(dev, 256, schedule)
    stream = torch.cuda.current_stream(dev)
    s = ctypes.c_void_p(stream.cuda_stream)

    ref = _outputs(req, dev)
    queue = torch.zeros((1,), dtype=torch.int64, device=dev)
    args = build_args(req, ref, queue, None)
    scratch = alloc_scratch(args, dev)
    assert lib.pb_solve_scratch_bytes(ctypes.byref(args)) + 256 <= L.NOALLOC_SCRATCH_BYTES
    L.check(lib.pb_solve_batch(ctypes.byref(args), s), "pb_solve_batch")
    torch.cuda.synchronize()
    del scratch

    for _ in range(2):
        out = _outputs(req, dev)
        a = build_args(req, out, None, None)  # no scratch, no queue counter: the library's own array is used
        rc = lib.pb_solve_batch_noalloc(ctypes.byref(a), s)
        assert rc == L.PB_SUCCESS, L.error_string(rc)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.status.cpu().numpy(), ref.status.cpu().numpy())
        np.testing.assert_array_equal(out.steps.cpu().numpy(), ref.steps.cpu().numpy())
        np.testing.assert_allclose(out.features.cpu().numpy(), ref.features.cpu().numpy(), rtol=1e-9, atol=0)
        np.testing.assert_allclose(out.y_final.cpu().numpy(), ref.y_final.cpu().numpy(), rtol=1e-6, atol=0)


def test_noalloc_refuses_requests_beyond_its_scratch():
    dev = torch.device("cuda:0")
    lib = L.load()
    req = _request(dev, 4)
    out = _outputs(req, dev)
    a = build_args(req, out, None, None)
    a.n_traj = 1_000_000  # step records of 1e6 trajectories do not fit the fixed array
    a.n_ic = 1_000_000
    assert lib.pb_solve_scratch_bytes(ctypes.byref(a)) + 256 > L.NOALLOC_SCRATCH_BYTES
    assert lib.pb_solve_batch_noalloc(ctypes.byref(a), None) == L.PB_ESCRATCH_LIMIT
    assert "fixed scratch" in L.error_string(L.PB_ESCRATCH_LIMIT)
