"""Coupled-oscillator networks: the Rössler network case study.

* :class:`RosslerNetworkODE` — params ``{a, b, c, K}`` plus an undirected edge
  list; state ``[x_0..x_{n-1}, y_0.., z_0..]`` (case_studies/rossler_network/
  rossler_network_jax_ode.py:53-79).  The reference's JAX class
  (``RosslerNetworkJaxODE``, with ``_N``, ``_edges_i``, ``_edges_j``) is accepted too.
* :func:`watts_strogatz` — a seeded small-world graph (ring of degree k, each
  edge rewired with probability p), the topology family of the case study.
* :class:`SyncFeatureExtractor` — the reference's ``SynchronizationFeatureExtractor``
  (synchronization_feature_extractor.py:73-106) over features the network
  kernel computes from the final state.
* :func:`sync_labels` — ``SynchronizationClassifier`` (synchronization_classifier.py:36-54)
  plus the unbounded class from the stop event.
"""

from __future__ import annotations

from typing import Any

import numpy as np
import torch

from pybasin_b200 import _lib as L
from pybasin_b200.engine import FeatureColumn
from pybasin_b200.odes import ODESystem

SYNC_NAMES = ["max_deviation_x", "max_deviation_y", "max_deviation_z", "max_deviation_all"]


def csr_from_edges(edges: np.ndarray, n: int) -> tuple[np.ndarray, np.ndarray]:
    """CSR adjacency (both directions of every undirected edge), neighbours sorted."""
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    if e.size and (e.min() < 0 or e.max() >= n):
        raise ValueError("edge endpoint outside [0, n)")
    src = np.concatenate([e[:, 0], e[:, 1]])
    dst = np.concatenate([e[:, 1], e[:, 0]])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    row = np.zeros(n + 1, dtype=np.int32)
    np.add.at(row, src + 1, 1)
    return np.cumsum(row).astype(np.int32), dst.astype(np.int32)


def watts_strogatz(n: int, k: int, p: float, seed: int) -> np.ndarray:
    """Undirected edges of a Watts–Strogatz graph: ring lattice of even degree k,
    each lattice edge (i, i+j) rewired to a uniform non-neighbour with probability p."""
    if k % 2 or k >= n:
        raise ValueError("k must be even and < n")
    rng = np.random.default_rng(seed)
    adj = [set() for _ in range(n)]
    for i in range(n):
        for j in range(1, k // 2 + 1):
            u, v = i, (i + j) % n
            adj[u].add(v)
            adj[v].add(u)
    for j in range(1, k // 2 + 1):
        for i in range(n):
            u, v = i, (i + j) % n
            if v not in adj[u] or rng.random() >= p:
                continue
            choices = [w for w in range(n) if w != u and w not in adj[u]]
            if not choices:
                continue
            w = int(rng.choice(choices))
            adj[u].discard(v)
            adj[v].discard(u)
            adj[u].add(w)
            adj[w].add(u)
    return np.array(sorted({(min(u, v), max(u, v)) for u in range(n) for v in adj[u]}), dtype=np.int32)


class RosslerNetworkODE(ODESystem):
    """Coupled Rössler oscillators with diffusive x-coupling on a graph."""

    b200_system = "rossler_network"

    def __init__(self, params: dict[str, float], n: int, edges: np.ndarray):
        super().__init__(params)
        self.n_nodes = n
        self.edges = np.asarray(edges, dtype=np.int32).reshape(-1, 2)
        self.csr = csr_from_edges(self.edges, n)

    def ode(self, t, y, p):
        n = self.n_nodes
        a, b, c, k = p[..., 0], p[..., 1], p[..., 2], p[..., 3]
        x, yy, z = y[..., :n], y[..., n : 2 * n], y[..., 2 * n :]
        row, col = (torch.as_tensor(v, device=y.device, dtype=torch.long) for v in self.csr)
        src = torch.repeat_interleave(torch.arange(n, device=y.device), row[1:] - row[:-1])
        lap = torch.zeros_like(x).index_add_(-1, src, x[..., col] - x[..., src])
        return torch.cat([-yy - z + k * lap, x + a * yy, b + z * (x - c)], dim=-1)


def network_csr(ode_system: Any) -> tuple[np.ndarray, np.ndarray, int]:
    """(row_ptr, col_idx, n_nodes) of a network ODE system (ours or the reference's JAX class)."""
    csr = getattr(ode_system, "csr", None)
    if csr is not None:
        return csr[0], csr[1], int(ode_system.n_nodes)
    n = int(getattr(ode_system, "_N"))
    ei = np.asarray(getattr(ode_system, "_edges_i"))
    ej = np.asarray(getattr(ode_system, "_edges_j"))
    # the reference stores both directions already (rossler_network_topology.py:build_edge_arrays)
    order = np.lexsort((ej, ei))
    ei, ej = ei[order], ej[order]
    row = np.zeros(n + 1, dtype=np.int32)
    np.add.at(row, ei + 1, 1)
    return np.cumsum(row).astype(np.int32), ej.astype(np.int32), n


class SyncFeatureExtractor:
    """Synchronisation features [max_dev_x, max_dev_y, max_dev_z, max_dev_all] at the final state."""

    def __init__(self, n_nodes: int, time_steady: float | None = None, device: str = "gpu"):
        self.n_nodes = n_nodes
        self.time_steady = time_steady
        self.device = device
        self.normalize = False

    def columns(self, num_states: int) -> list[FeatureColumn]:
        if num_states != 3 * self.n_nodes:
            raise ValueError(f"state has {num_states} components, expected 3 x {self.n_nodes}")
        return [FeatureColumn(i, L.FEAT_SYNC_DEV, 0.0, SYNC_NAMES[i]) for i in range(4)]

    def resolve_time_steady(self, save_ts: torch.Tensor) -> float:
        return float(save_ts[-1])

    def extract_features(self, solution: Any) -> torch.Tensor:
        feats = getattr(solution.y, "_pb_features", None)
        if feats is None:
            raise RuntimeError("SyncFeatureExtractor reads features computed inside B200Dopri5Solver")
        return feats

    @property
    def feature_names(self) -> list[str]:
        return list(SYNC_NAMES)


def sync_labels(features: torch.Tensor, status: torch.Tensor, epsilon: float = 1.5) -> np.ndarray:
    """'synchronized' if max_dev_all < epsilon, else 'desynchronized'; 'unbounded' after a stop."""
    f = features[:, 3].detach().cpu().numpy()
    st = status.detach().cpu().numpy()
    lab = np.where(f < epsilon, "synchronized", "desynchronized").astype(object)
    lab[st == L.TRAJ_UNBOUNDED] = "unbounded"
    return lab
