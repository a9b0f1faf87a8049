"""Host-side layout of the fused training step (no GPU needed): the geometry the
library reports for a network, and which networks the fused step takes."""

from __future__ import annotations

import ctypes

import pytest

from pybasin_b200.train import _lib, fused_supported


def _geometry(dims: list[int], batch: int) -> list[int]:
    lib = _lib()
    n = len(dims) - 1
    d = (ctypes.c_int32 * len(dims))(*dims)
    out = (ctypes.c_int64 * (3 + 4 * n))()
    rc = lib.pb_train_fused_geometry(n, d, batch, out, len(out))
    assert rc == 0
    return list(out)


def test_surrogate_geometry():
    """136 -> 256 x4 -> 6: inputs augmented by the ones column to 144 / 272, the
    six classes padded to 16 rows; the images (the augmented weights, and W^T of
    every layer after the first for the input gradients) and the scratch sized
    from those."""
    dims = [136, 256, 256, 256, 256, 6]
    g = _geometry(dims, 4096)
    kaug = [g[3 + 4 * l] for l in range(5)]
    npad = [g[4 + 4 * l] for l in range(5)]
    aug_off = [g[5 + 4 * l] for l in range(5)]
    w_off = [g[6 + 4 * l] for l in range(5)]
    assert kaug == [144, 272, 272, 272, 272] and npad == [256, 256, 256, 256, 16]
    sizes = [n * k for n, k in zip(npad, kaug)]
    wt = [0] + [dims[l] * npad[l] for l in range(1, 5)]  # W^T: d_in x npad
    assert g[2] == sum(sizes) and g[0] == 2 * (sum(sizes) + sum(wt))
    assert aug_off == [sum(sizes[:l]) for l in range(5)]
    assert w_off == [2 * (sum(sizes[:l]) + sum(wt[:l])) for l in range(5)]
    tiles = 4096 // 128
    per_tile = sum(128 * k * 2 + 128 * n * 2 for k, n in zip(kaug, npad)) + 4 * 128 * 256 * 2
    assert g[1] == tiles * per_tile


@pytest.mark.parametrize("dims,ok", [([136, 256, 256, 6], True), ([24, 64, 6], True), ([20, 64, 6], False),
                                     ([24, 72, 6], False), ([24, 64, 33], False), ([24, 512, 6], False),
                                     ([8, 2], True), ([24] + [64] * 8 + [4], False)])
def test_fused_limits(dims, ok):
    assert fused_supported(dims) == ok
    lib = _lib()
    n = len(dims) - 1
    d = (ctypes.c_int32 * len(dims))(*dims)
    out = (ctypes.c_int64 * (3 + 4 * max(n, 1)))()
    rc = lib.pb_train_fused_geometry(n, d, 256, out, len(out))
    assert (rc == 0) == ok


def test_geometry_rejects_a_short_output_array():
    lib = _lib()
    d = (ctypes.c_int32 * 3)(24, 64, 6)
    out = (ctypes.c_int64 * 5)()
    assert lib.pb_train_fused_geometry(2, d, 256, out, len(out)) != 0
