"""Parameter-study batching: many parameter points with uneven IC counts in one launch.

The reference's parameter study integrates B ICs against every parameter row
(IC-major expansion, src/pybasin/solvers/base.py:155-159); here each IC carries
its own parameter point, so points can have different sample counts, and the
whole study is one integrator launch plus one labelling launch (graph-capturable).
Labels are checked per point against the FP64 oracle + the reference's 1-NN.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.helpers import PENDULUM, knn_labels, seeded_ics

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _sweep(n_points: int, lo: int, hi: int):
    rng = np.random.default_rng(42)
    T = np.linspace(0.1, 1.0, n_points)
    n_p = np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), n_points))).astype(int)
    ics = [seeded_ics(PENDULUM, int(k), seed=42 + p) for p, k in enumerate(n_p)]
    y0 = torch.cat(ics)
    group = torch.cat([torch.full((int(k),), p, dtype=torch.int32) for p, k in enumerate(n_p)])
    rows = np.array([[0.1, t, 1.0] for t in T])
    return rows, n_p, y0, group


def _pipeline(precision: str, rows: np.ndarray):
    from pybasin_b200 import B200Dopri5Solver, FusedFeatureExtractor, PendulumODE
    from pybasin_b200.pipeline import BasinStabilityPipeline

    fx = FusedFeatureExtractor(time_steady=950.0, features=None, features_per_state={1: {"log_delta": None}},
                               normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=1000, device="cuda:0", precision=precision,
                              feature_extractor=fx)
    return BasinStabilityPipeline(PendulumODE({"alpha": 0.1, "T": 0.5, "K": 1.0}), solver,
                                  [list(t) for t in PENDULUM.templates], list(PENDULUM.classes), device=DEV,
                                  param_rows=rows)


def _oracle_labels(rows, y0, group):
    save = PENDULUM.save_ts().numpy()
    feats = [(1, 9, 0.0)]
    r = O.solve_batch(O.SYS_PENDULUM, y0.double().numpy(), rows, save, (0.0, 1000.0), 1e-8, 1e-6,
                      param_index=group.numpy(), win_begin=PENDULUM.win_begin(), features=feats)
    rt = O.solve_batch(O.SYS_PENDULUM, np.array(PENDULUM.templates), np.array([PENDULUM.params]), save, (0.0, 1000.0),
                       1e-8, 1e-6, win_begin=PENDULUM.win_begin(), features=feats)
    return knn_labels(rt["features"], r["features"])


@pytest.mark.parametrize("precision,max_flips", [("fp64", 2), ("mixed", 6)])
def test_pendulum_torque_sweep_in_one_launch(precision, max_flips):
    rows, n_p, y0, group = _sweep(16, 100, 800)
    pipe = _pipeline(precision, rows)
    labels, counts = pipe.run_device(y0.to(DEV), group=group.to(DEV))
    torch.cuda.synchronize()
    lab = labels.cpu().numpy()
    cnt = counts.cpu().numpy()
    want = _oracle_labels(rows, y0, group)
    g = group.numpy()
    for p in range(len(n_p)):
        sel = g == p
        assert cnt[p].sum() == n_p[p]
        np.testing.assert_array_equal(cnt[p, :2], np.bincount(lab[sel], minlength=2))
        assert (lab[sel] != want[sel]).sum() <= max_flips, f"point {p}: T={rows[p, 1]:.3f}"
    # T >= K leaves no fixed point: every IC rotates
    assert cnt[-1, 0] == 0


def test_sweep_graph_replay_matches_eager():
    rows, n_p, y0, group = _sweep(8, 50, 300)
    pipe = _pipeline("mixed", rows)
    lab_e, cnt_e = pipe.run_device(y0.to(DEV), group=group.to(DEV))
    lab_e, cnt_e = lab_e.clone(), cnt_e.clone()
    lab_g, cnt_g = pipe.run_device(y0.to(DEV), group=group.to(DEV), use_graph=True)
    lab_g2, cnt_g2 = pipe.run_device(y0.to(DEV), group=group.to(DEV), use_graph=True)
    torch.cuda.synchronize()
    assert torch.equal(lab_e, lab_g) and torch.equal(cnt_e, cnt_g)
    assert torch.equal(lab_g, lab_g2) and torch.equal(cnt_g, cnt_g2)


def test_lorenz_rho_sweep_with_unbounded_threshold():
    """Lorenz sigma=10, beta=8/3, rho in {0.5, 15, 28}, ICs U[-20,20]^3, stop at |y| > 1e6."""
    from pybasin_b200 import _lib as L
    from pybasin_b200.engine import FeatureColumn, SolveRequest, solve

    rng = np.random.default_rng(3)
    per = 200
    y0 = rng.uniform(-20, 20, (3 * per, 3))
    rows = np.array([[10.0, rho, 8.0 / 3.0] for rho in (0.5, 15.0, 28.0)])
    group = np.repeat(np.arange(3), per).astype(np.int32)
    save = np.linspace(150.0, 200.0, 501)
    feats = [(0, L.FEAT_MEAN, 0.0), (2, L.FEAT_MEAN, 0.0), (0, L.FEAT_STD, 0.0)]
    want = O.solve_batch(O.SYS_LORENZ, y0, rows, save, (0.0, 200.0), 1e-8, 1e-6, param_index=group,
                         features=feats, unbounded_thr=1e6)
    req = SolveRequest(system=L.SYS_LORENZ, dim=3, y0=torch.tensor(y0, device=DEV),
                       params=torch.tensor(rows, device=DEV), save_ts=torch.tensor(save, device=DEV),
                       t_span=(0.0, 200.0), rtol=1e-8, atol=1e-6, layout=L.LAYOUT_INDEXED,
                       param_index=torch.tensor(group, device=DEV), columns=[FeatureColumn(*f) for f in feats],
                       unbounded_thr=1e6, precision=L.PREC_FP64)
    r = solve(req)
    torch.cuda.synchronize()
    st = r.status.cpu().numpy()
    f = r.features.cpu().numpy()
    assert (st == 0).all() and (want["status"] == 0).all()  # the classic system stays bounded
    # rho = 0.5 (origin) and rho = 15 (C+/C-) converge: features agree
    conv = group < 2
    np.testing.assert_allclose(f[conv][:, :2], want["features"][conv][:, :2], rtol=1e-5, atol=1e-6)
    # rho = 28 is chaotic: pointwise values decorrelate; the attractor's statistics agree
    chaos = group == 2
    assert abs(f[chaos][:, 1].mean() - want["features"][chaos][:, 1].mean()) < 0.5


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("dim", [1, 2, 3, 5])
def test_device_morton_keys_match_host_statement(dtype, dim):
    from pybasin_b200.engine import MortonOrder, morton_keys

    g = torch.Generator().manual_seed(dim)
    y0 = (torch.rand(20_011, dim, generator=g, dtype=torch.float64) * 7.0 - 3.0).to(dtype)
    groups = torch.randint(0, 9, (20_011,), generator=g, dtype=torch.int32)
    mo = MortonOrder(torch.device("cuda:0"))
    for grp in (None, groups):
        want = morton_keys(y0, groups=grp)
        got = mo.keys_of(y0.cuda(), groups=None if grp is None else grp.cuda()).cpu()
        assert torch.equal(got, want)
    # a constant coordinate (zero span)
    y1 = y0.clone()
    y1[:, 0] = 1.5
    assert torch.equal(mo.keys_of(y1.cuda()).cpu(), morton_keys(y1))


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_device_order_is_the_stable_argsort_of_the_keys(dim):
    """pb_morton_order (radix sort over the key bits in use) against torch's stable
    argsort of the same keys, with and without groups, duplicate keys included."""
    from pybasin_b200.engine import MortonOrder

    g = torch.Generator().manual_seed(7 + dim)
    y0 = torch.rand(30_001, dim, generator=g) * 4.0 - 2.0
    y0[1000:1100] = y0[5]  # equal keys keep their index order
    groups = torch.randint(0, 5, (30_001,), generator=g, dtype=torch.int32)
    mo = MortonOrder(torch.device("cuda:0"))
    for grp in (None, groups.cuda()):
        keys = mo.keys_of(y0.cuda(), groups=grp).clone()
        want = torch.argsort(keys, stable=True).to(torch.int32)
        got = mo(y0.cuda(), groups=grp)
        assert torch.equal(got, want)
    out = torch.full((30_001,), -1, dtype=torch.int32, device="cuda:0")
    assert mo(y0.cuda(), out=out) is out and torch.equal(out, torch.argsort(mo.keys_of(y0.cuda()).clone(), stable=True).to(torch.int32))


@pytest.mark.gpu
def test_device_order_of_tiny_and_empty_inputs():
    from pybasin_b200.engine import MortonOrder

    mo = MortonOrder(torch.device("cuda:0"))
    assert mo(torch.zeros((0, 2), device="cuda:0")).numel() == 0
    one = mo(torch.tensor([[0.5, -0.25]], device="cuda:0"))
    assert one.tolist() == [0]
    same = mo(torch.ones((5, 3), device="cuda:0"))  # equal keys: the identity, in index order
    assert same.tolist() == [0, 1, 2, 3, 4]
