"""Parameter studies at their full sizes (pybasin_b200/studies.py), one launch each.

Per parameter point, the mixed kernel's class fractions against the plain FP64
kernel's on the same ICs (|dBS| <= 0.005 where trajectories are not chaotic),
and the FP64 kernel's labels against the FP64 oracle on a seeded subsample of
every point.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pybasin_b200 import _lib as L
from pybasin_b200 import studies as S
from tests.helpers import PENDULUM, knn_labels

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def test_pendulum_torque_sweep_at_full_size():
    """64 torque points, 1k-50k ICs each (about 0.8 M), one graph-captured launch."""
    st = S.pendulum_torque_sweep()
    n = st.y0.shape[0]
    assert len(st.counts) == 64 and 600_000 <= n <= 1_000_000 and st.counts.min() >= 1000
    y0, group = st.y0.to(DEV), st.group.to(DEV)
    mixed = S.pendulum_pipeline("mixed", st.rows, DEV)
    lab_m, cnt_m = mixed.run_device(y0, group=group, use_graph=True)
    lab_m, cnt_m = lab_m.clone(), cnt_m.clone()
    fp64 = S.pendulum_pipeline("fp64", st.rows, DEV)
    lab_d, cnt_d = fp64.run_device(y0, group=group)
    torch.cuda.synchronize()
    cm, cd = cnt_m.cpu().numpy(), cnt_d.cpu().numpy()
    assert (cm.sum(axis=1) == st.counts).all() and (cd.sum(axis=1) == st.counts).all()
    dbs = np.abs(cm[:, :2] - cd[:, :2]).max(axis=1) / st.counts
    assert dbs.max() <= 0.005, f"point {dbs.argmax()}: |dBS| {dbs.max():.4f}"
    assert cd[-1, 0] == 0  # T = K: no fixed point, every IC rotates
    # the FP64 kernel against the oracle on 40 ICs of every point
    g = st.group.numpy()
    pick = np.concatenate([np.nonzero(g == p)[0][:40] for p in range(64)])
    save = PENDULUM.save_ts().numpy()
    r = O.solve_batch(O.SYS_PENDULUM, st.y0[pick].double().numpy(), st.rows, save, (0.0, 1000.0), 1e-8, 1e-6,
                      param_index=g[pick], win_begin=PENDULUM.win_begin(), features=[(1, 9, 0.0)])
    rt = O.solve_batch(O.SYS_PENDULUM, np.array(PENDULUM.templates), np.array([PENDULUM.params]), save, (0.0, 1000.0),
                       1e-8, 1e-6, win_begin=PENDULUM.win_begin(), features=[(1, 9, 0.0)])
    want = knn_labels(rt["features"], r["features"])
    got = lab_d.cpu().numpy()[pick]
    assert (got != want).sum() <= 3


def test_lorenz_rho_sweep_at_full_size():
    """rho in {0.5, 15, 28}, 20,000 ICs each on [-20, 20]^3, one launch per precision."""
    st = S.lorenz_rho_sweep(20_000)
    rm = S.lorenz_solve(st, L.PREC_MIXED, DEV)
    rd = S.lorenz_solve(st, L.PREC_FP64, DEV)
    torch.cuda.synchronize()
    g = st.group.to(DEV)
    lm = S.lorenz_labels(rm.features, rm.status)
    ld = S.lorenz_labels(rd.features, rd.status)
    fm = S.per_point_fractions(lm, g, 3, 5).cpu().numpy()
    fd = S.per_point_fractions(ld, g, 3, 5).cpu().numpy()
    assert (rd.status.cpu().numpy() == 0).all()  # the classic system stays bounded
    assert fd[0, 0] == 1.0  # rho = 0.5: the origin
    assert fd[1, 1] > 0.3 and fd[1, 2] > 0.3 and fd[1, 1] + fd[1, 2] == 1.0  # rho = 15: C+ and C-
    assert fd[2, 3] == 1.0  # rho = 28: the butterfly
    # converging points: class fractions within 0.005 of FP64; the chaotic one is one class
    assert np.abs(fm[:2] - fd[:2]).max() <= 0.005
    assert fm[2, 3] == 1.0
    # FP64 kernel vs the oracle on 30 ICs of each converging point (mean and spread of x)
    gg = st.group.numpy()
    pick = np.concatenate([np.nonzero(gg == p)[0][:30] for p in (0, 1)])
    save = torch.linspace(900.0, 1000.0, 1000, dtype=torch.float32).double().numpy()
    w = O.solve_batch(O.SYS_LORENZ, st.y0[pick].double().numpy(), st.rows, save, (0.0, 1000.0), 1e-8, 1e-6,
                      param_index=gg[pick], features=[(0, 1, 0.0), (0, 2, 0.0)], unbounded_thr=1e6)
    np.testing.assert_allclose(rd.features.cpu().numpy()[pick], w["features"], rtol=1e-6, atol=1e-6)


def test_rossler_coupling_sweep_at_full_size():
    """8 couplings x 20,000 ICs of the 100-node network (300 states each) in one
    launch; the mixed kernel's synchronisation labels against the FP64 kernel's on
    2,000 ICs of every coupling."""
    st, csr = S.rossler_coupling_sweep(20_000)
    rm = S.rossler_solve(st, csr, L.PREC_MIXED, DEV)
    torch.cuda.synchronize()
    g = st.group.to(DEV)
    lm = S.rossler_labels(rm.features, rm.status)
    fm = S.per_point_fractions(lm, g, 8, 3).cpu().numpy()
    assert set(np.unique(rm.status.cpu().numpy())) <= {L.TRAJ_OK, L.TRAJ_UNBOUNDED}
    # the FP64 kernel on the first 2,000 ICs of every coupling
    gg = st.group.numpy()
    pick = torch.tensor(np.concatenate([np.nonzero(gg == p)[0][:2000] for p in range(8)]))
    sub = S.Study(st.y0[pick], st.group[pick], st.rows, np.full(8, 2000))
    rd = S.rossler_solve(sub, csr, L.PREC_FP64, DEV)
    torch.cuda.synchronize()
    ld = S.rossler_labels(rd.features, rd.status).cpu()
    agree = (ld == lm.cpu()[pick]).double().mean().item()
    assert agree >= 0.97
    fd = S.per_point_fractions(ld, sub.group, 8, 3).numpy()
    fm_sub = S.per_point_fractions(lm.cpu()[pick], sub.group, 8, 3).numpy()
    assert np.abs(fm_sub - fd).max() <= 0.03
    # stronger coupling synchronises more of the bounded trajectories
    sync_share = fm[:, 0] / np.maximum(fm[:, 0] + fm[:, 1], 1e-12)
    assert sync_share[-1] >= sync_share[0]
