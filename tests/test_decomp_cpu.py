"""Slab decomposition bookkeeping (athena_cuda_b200/decomp.py): the rows of
each rank, its neighbours and which x2 sides take the physical boundary."""
from __future__ import annotations

import pytest

from athena_cuda_b200.decomp import NG, neighbours, slab_rows, x2_sides


def test_slab_rows_cover_the_grid_once():
    for nx2, ranks in [(64, 1), (64, 2), (67, 3), (300, 8), (40, 10)]:
        s = slab_rows(nx2, ranks)
        assert sum(n for _, n in s) == nx2
        assert [j0 for j0, _ in s] == [sum(n for _, n in s[:r]) for r in range(ranks)]
        assert max(n for _, n in s) - min(n for _, n in s) <= 1
        assert min(n for _, n in s) >= NG
    with pytest.raises(ValueError):
        slab_rows(12, 4)  # slabs thinner than the ghost depth


def test_neighbours_and_physical_sides():
    assert neighbours(0, 1, True) == (None, None) and x2_sides(0, 1, True) == 3
    assert neighbours(0, 3, True) == (2, 1) and neighbours(2, 3, True) == (1, 0)
    assert all(x2_sides(r, 3, True) == 0 for r in range(3))
    assert neighbours(0, 3, False) == (None, 1) and neighbours(2, 3, False) == (1, None)
    assert [x2_sides(r, 3, False) for r in range(3)] == [1, 0, 2]
    assert neighbours(0, 2, True) == (1, 1)


def test_transport_is_checked_before_any_device_work():
    from athena_cuda_b200 import configs
    from athena_cuda_b200.decomp import MAX_RANKS, SlabGrid

    with pytest.raises(ValueError, match="transport"):
        SlabGrid(configs.blast(16, 16), "blast", 0, 2, transport="tcp")
    with pytest.raises(ValueError, match="at most"):
        SlabGrid(configs.blast(16, 16 * (MAX_RANKS + 1)), "blast", 0, MAX_RANKS + 1, transport="ipc")
