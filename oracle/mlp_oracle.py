"""FP64 NumPy restatement of the surrogate MLP (forward, softmax cross-entropy, backward).

TEST INFRASTRUCTURE ONLY: the checker for the BF16 tensor-core kernels of
pybasin_b200/csrc/pb_mlp.cu (tests/test_surrogate.py).  Layers: h = GELU(x W^T + b)
for the hidden layers (GELU in its tanh form, evaluated exactly in FP64),
logits = h W^T + b for the last one.
"""

from __future__ import annotations

import numpy as np

_A = np.sqrt(2.0 / np.pi)
_B = 0.044715


def gelu(z: np.ndarray) -> np.ndarray:
    """0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    return 0.5 * z * (1.0 + np.tanh(_A * (z + _B * z**3)))


def gelu_grad(z: np.ndarray) -> np.ndarray:
    t = np.tanh(_A * (z + _B * z**3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _A * (1.0 + 3.0 * _B * z * z)


def forward(x: np.ndarray, Ws: list[np.ndarray], bs: list[np.ndarray]):
    acts, pres = [x], []
    h = x
    for i, (W, b) in enumerate(zip(Ws, bs)):
        z = h @ W.T + b
        if i == len(Ws) - 1:
            return z, acts, pres
        pres.append(z)
        h = gelu(z)
        acts.append(h)
    raise AssertionError


def loss_and_grad(logits: np.ndarray, y: np.ndarray):
    m = logits.max(axis=1, keepdims=True)
    e = np.exp(logits - m)
    p = e / e.sum(axis=1, keepdims=True)
    n = logits.shape[0]
    loss = -np.log(p[np.arange(n), y]).sum()
    d = p.copy()
    d[np.arange(n), y] -= 1.0
    return loss, d / n


def backward(dlogits: np.ndarray, acts, pres, Ws):
    gW = [None] * len(Ws)
    gb = [None] * len(Ws)
    dz = dlogits
    for i in reversed(range(len(Ws))):
        gW[i] = dz.T @ acts[i]
        gb[i] = dz.sum(axis=0)
        if i == 0:
            break
        dz = (dz @ Ws[i]) * gelu_grad(pres[i - 1])
    return gW, gb
