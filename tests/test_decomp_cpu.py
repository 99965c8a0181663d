"""Slab decomposition bookkeeping (athena_cuda_b200/decomp.py): the rows of
each rank, its neighbours and which x2 sides take the physical boundary."""
from __future__ import annotations

import pytest

from athena_cuda_b200.decomp import NG, block_neighbours, neighbours, slab_rows, x2_sides


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


def test_block_neighbours_2d():
    # 3 x 2 blocks, periodic in x1, walls in x2: rank = rx + 3 ry
    nb = block_neighbours(4, 3, 2, True, False)      # rx = 1, ry = 1
    assert nb[0] == (3, 5) and nb[1] == (1, None)
    assert nb["sides1"] == 0 and nb["sides2"] == 2
    nb = block_neighbours(0, 3, 2, True, False)
    assert nb[0] == (2, 1) and nb[1] == (None, 3) and nb["sides2"] == 1
    # one block across x1: its x1 ghosts are its own (periodic fill)
    nb = block_neighbours(1, 1, 2, True, True)
    assert nb[0] == (None, None) and nb["sides1"] == 3 and nb[1] == (0, 0) and nb["sides2"] == 0
    # every low/high pair is mutual
    for px, py in ((2, 2), (3, 2), (2, 3), (4, 1)):
        for r in range(px * py):
            nb = block_neighbours(r, px, py, True, True)
            for d in (0, 1):
                lo, hi = nb[d]
                assert (lo is None) == (hi is None) == ((px, py)[d] == 1)
                if lo is not None:
                    assert block_neighbours(lo, px, py, True, True)[d][1] == r
                    assert block_neighbours(hi, px, py, True, True)[d][0] == r


def test_one_sided_periodic_direction_is_not_split():
    from athena_cuda_b200 import configs
    from athena_cuda_b200.decomp import BlockGrid

    with pytest.raises(ValueError, match="periodic on both sides"):
        BlockGrid(configs.blast(32, 32, bc=(2, 4, 4, 4)), "blast", 0, 2, 1, transport="ipc")
