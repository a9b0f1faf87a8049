"""Rössler network (100 nodes, 300-dim state): one warp per trajectory.

Parity: FP64 kernel vs the FP64 oracle on a short horizon (rtol 1e-7 on the
final state); synchronisation labels of the mixed kernel vs the FP64 kernel;
and the reference's own paper-value test (tests/integration/rossler_network/
test_rossler_network.py:34-140): bounded basin stability per coupling K against
the published values with z = |A - B| / sqrt(SE_A^2 + SE_B^2) < 3.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pybasin_b200 import _lib as L
from pybasin_b200.engine import FeatureColumn, SolveRequest, solve
from pybasin_b200.network import csr_from_edges, watts_strogatz

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
GOLDEN = Path(__file__).resolve().parent / "golden"
N_NODES = 100


def _graph():
    g = np.load(GOLDEN / "rossler_network_reference.npz")
    return csr_from_edges(g["edges"], N_NODES), g


def _ics(n: int, seed: int) -> torch.Tensor:
    """UniformRandomSampler over x,y in [-15,15], z in [-5,35] per node (setup_rossler_network_system.py)."""
    lo = torch.tensor([-15.0] * N_NODES + [-15.0] * N_NODES + [-5.0] * N_NODES)
    hi = torch.tensor([15.0] * N_NODES + [15.0] * N_NODES + [35.0] * N_NODES)
    torch.manual_seed(seed)
    return torch.rand(n, 3 * N_NODES) * (hi - lo) + lo


def _solve(y0, params, csr, t1, rtol, atol, precision, save=None, group=None, unb=400.0, keep_final=True):
    feats = [FeatureColumn(i, L.FEAT_SYNC_DEV) for i in range(4)]
    save_ts = torch.tensor(save if save is not None else [t1], dtype=torch.float64, device=DEV)
    req = SolveRequest(system=L.SYS_ROSSLER_NET, dim=3 * N_NODES, y0=y0.to(DEV),
                       params=torch.tensor(np.atleast_2d(params), dtype=torch.float64, device=DEV), save_ts=save_ts,
                       t_span=(0.0, t1), rtol=rtol, atol=atol, columns=feats, precision=precision,
                       unbounded_thr=unb, keep_final=keep_final, out_dtype=torch.float64, keep_steps=True,
                       layout=L.LAYOUT_INDEXED if group is not None else L.LAYOUT_SINGLE,
                       param_index=None if group is None else torch.as_tensor(group, dtype=torch.int32, device=DEV),
                       csr_row=torch.tensor(csr[0], device=DEV), csr_col=torch.tensor(csr[1], device=DEV))
    r = solve(req)
    torch.cuda.synchronize()
    return r


def test_fp64_network_matches_oracle_short_horizon():
    csr, _ = _graph()
    # ICs near the attractor (x, y in [-5, 5], z in [0, 2]); from the sampler's full box
    # many trajectories blow up in finite time, which the unbounded test covers
    y0 = _ics(16, 1).double()
    y0[:, : 2 * N_NODES] /= 3.0
    y0[:, 2 * N_NODES :] = (y0[:, 2 * N_NODES :] + 5.0) / 20.0
    p = np.array([[0.2, 0.2, 7.0, 0.218]])
    # threshold off: every trajectory runs to t1 and is compared in full
    r = _solve(y0, p, csr, 5.0, 1e-9, 1e-9, L.PREC_FP64, unb=0.0)
    want = O.solve_batch(O.SYS_ROSSLER_NET, y0.numpy(), p, np.array([5.0]), (0.0, 5.0), 1e-9, 1e-9, csr=csr)
    assert (r.status.cpu().numpy() == 0).all() and (want["status"] == 0).all()
    # the warp-reduced error norm sums in another order: a marginal accept may flip
    assert np.abs(r.steps.cpu().numpy() - want["steps"]).max() <= 2
    np.testing.assert_allclose(r.y_final.cpu().numpy(), want["y_final"], rtol=1e-7, atol=1e-7)
    # features: max - min over nodes at the final state
    yf = want["y_final"].reshape(16, 3, N_NODES)
    dev = yf.max(axis=2) - yf.min(axis=2)
    f = r.features.cpu().numpy()
    np.testing.assert_allclose(f[:, :3], dev, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(f[:, 3], dev.max(axis=1), rtol=1e-6, atol=1e-6)


def test_unbounded_stop_matches_oracle():
    csr, _ = _graph()
    y0 = _ics(64, 5).double()
    p = np.array([[0.2, 0.2, 7.0, 0.218]])
    r = _solve(y0, p, csr, 20.0, 1e-8, 1e-8, L.PREC_FP64, unb=400.0)
    want = O.solve_batch(O.SYS_ROSSLER_NET, y0.numpy(), p, np.array([20.0]), (0.0, 20.0), 1e-8, 1e-8, csr=csr,
                         unbounded_thr=400.0)
    st = r.status.cpu().numpy()
    assert (st == L.TRAJ_UNBOUNDED).any() and (st == L.TRAJ_OK).any()
    np.testing.assert_array_equal(st, want["status"])
    f = r.features.cpu().numpy()
    assert np.isinf(f[st == L.TRAJ_UNBOUNDED]).all() and np.isfinite(f[st == L.TRAJ_OK]).all()


def test_mixed_network_labels_agree_with_fp64():
    csr, _ = _graph()
    y0 = _ics(512, 2)
    p = np.array([[0.2, 0.2, 7.0, 0.218]])
    r64 = _solve(y0, p, csr, 1000.0, 1e-3, 1e-6, L.PREC_FP64, save=np.linspace(980, 1000, 200))
    r32 = _solve(y0, p, csr, 1000.0, 1e-3, 1e-6, L.PREC_MIXED, save=np.linspace(980, 1000, 200))

    def lab(r):
        st = r.status.cpu().numpy()
        f = r.features.cpu().numpy()[:, 3]
        return np.where(st == L.TRAJ_UNBOUNDED, 2, np.where(f < 1.5, 0, 1))

    a, b = lab(r64), lab(r32)
    assert (a == b).mean() >= 0.97
    assert abs((a == 2).mean() - (b == 2).mean()) <= 0.02


def test_bounded_basin_stability_matches_paper_values():
    """The reference's paper validation, all 11 K values in one launch (per-IC parameter rows)."""
    csr, g = _graph()
    ks, sb = g["k_values"], g["expected_sb"]
    n_per = 800
    y0 = _ics(n_per * len(ks), 42)
    rows = np.array([[0.2, 0.2, 7.0, k] for k in ks])
    group = np.repeat(np.arange(len(ks)), n_per)
    r = _solve(y0, rows, csr, 1000.0, 1e-3, 1e-6, L.PREC_MIXED, save=np.linspace(980, 1000, 200), group=group,
               keep_final=False)
    st = r.status.cpu().numpy()
    assert set(np.unique(st)) <= {L.TRAJ_OK, L.TRAJ_UNBOUNDED}
    n_ref = int(g["n_reference"])
    for i, (k, want) in enumerate(zip(ks, sb)):
        got = float((st[group == i] != L.TRAJ_UNBOUNDED).mean())
        se = np.sqrt(got * (1 - got) / n_per + want * (1 - want) / n_ref)
        z = abs(got - want) / se
        assert z < 3.0, f"K={k}: S_B {got:.3f} vs paper {want:.3f} (z={z:.2f})"


def test_seeded_watts_strogatz_graph():
    e = watts_strogatz(100, 4, 0.1, seed=42)
    assert len(e) == 200  # rewiring keeps the edge count n*k/2
    assert (e[:, 0] < e[:, 1]).all()
    assert np.array_equal(e, watts_strogatz(100, 4, 0.1, seed=42))
    row, col = csr_from_edges(e, 100)
    assert row[-1] == 400 and col.max() < 100


def test_invalid_graph_is_reported_not_read():
    csr, _ = _graph()
    bad_col = csr[1].copy()
    bad_col[5] = 1000  # a neighbour outside the graph
    r = _solve(_ics(4, 3), np.array([[0.2, 0.2, 7.0, 0.2]]), (csr[0], bad_col), 1.0, 1e-3, 1e-6, L.PREC_MIXED)
    assert (r.status.cpu().numpy() == L.TRAJ_BAD_INPUT).all()


def test_solver_drop_in_with_sync_extractor():
    """B200Dopri5Solver.integrate on a network ODE object, features read by SyncFeatureExtractor."""
    from pybasin_b200 import B200Dopri5Solver
    from pybasin_b200.network import RosslerNetworkODE, SyncFeatureExtractor, sync_labels

    csr, g = _graph()
    ode = RosslerNetworkODE({"a": 0.2, "b": 0.2, "c": 7.0, "K": 0.218}, N_NODES, g["edges"])
    ext = SyncFeatureExtractor(N_NODES)
    solver = B200Dopri5Solver(t_span=(0, 200), t_steps=200, device="cuda", rtol=1e-3, atol=1e-6,
                              precision="mixed", feature_extractor=ext, unbounded_threshold=400.0)
    y0 = _ics(256, 9)
    t, y = solver.integrate(ode, y0)
    feats = ext.extract_features(types_ns(y))
    assert feats.shape == (256, 4) and t.shape == (1,)
    direct = _solve(y0, np.array([[0.2, 0.2, 7.0, 0.218]]), csr, 200.0, 1e-3, 1e-6, L.PREC_MIXED,
                    save=np.linspace(0, 200, 200), keep_final=False)
    # same kernel, same inputs: identical features and statuses (processing order does not matter)
    np.testing.assert_array_equal(feats.cpu().numpy(), direct.features.float().cpu().numpy())
    lab = sync_labels(feats, y._pb_status)
    assert set(lab) <= {"synchronized", "desynchronized", "unbounded"}


def types_ns(y):
    from types import SimpleNamespace

    return SimpleNamespace(y=y)
