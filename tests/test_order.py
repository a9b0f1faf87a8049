"""Z-order processing order (host statement of pb_morton_keys)."""

from __future__ import annotations

import torch

from pybasin_b200.engine import morton_keys, spatial_order


def test_unit_square_corners_interleave_x_then_y():
    y0 = torch.tensor([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]])
    assert morton_keys(y0, bits=1).tolist() == [0, 1, 2, 3]
    assert morton_keys(y0, bits=2).tolist() == [0, 5, 10, 15]


def test_group_major_keys_and_permutation():
    g = torch.Generator().manual_seed(3)
    y0 = torch.rand(1000, 2, generator=g)
    groups = torch.randint(0, 4, (1000,), generator=g)
    order = spatial_order(y0, groups=groups)
    assert sorted(order.tolist()) == list(range(1000))
    assert (groups[order.long()].diff() >= 0).all()  # group-major
    # within a group, consecutive positions are spatial neighbours more often than random pairs
    o = order.long()
    step = (y0[o[1:]] - y0[o[:-1]]).norm(dim=1).median()
    rand = (y0[torch.randperm(1000, generator=g)] - y0).norm(dim=1).median()
    assert step < 0.25 * rand


def test_empty_and_zero_span():
    assert spatial_order(torch.zeros((0, 3))).numel() == 0
    y0 = torch.ones((5, 3))
    assert morton_keys(y0).tolist() == [0] * 5
