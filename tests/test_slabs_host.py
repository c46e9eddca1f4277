"""The slab decomposition's host logic: the split of the planes over parts (the rule fvg_create_part applies) and the
split / join of states in the reference's cell order."""
import numpy as np
import pytest

from fenice_b200 import slabs


@pytest.mark.parametrize("n,nparts", [(13, 3), (256, 8), (9, 2), (10, 10)])
def test_part_ranges_tile_the_axis(n, nparts):
    ranges = [slabs.part_range(n, nparts, p) for p in range(nparts)]
    assert ranges[0][0] == 0
    for (f0, c0), (f1, _) in zip(ranges, ranges[1:]):
        assert f1 == f0 + c0
    assert sum(c for _, c in ranges) == n
    assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1


@pytest.mark.parametrize("shape", [(7, 5, 9), (6, 11, 1)])
def test_split_join_round_trip(shape):
    nx, ny, nz = shape
    params = dict(nx=nx, ny=ny, nz=nz)
    U = np.arange(nx * ny * nz * 5, dtype=np.float64).reshape(-1, 5)
    parts = slabs.split_state(params, U, 3)
    ax = slabs.split_axis(params)
    n = nz if ax == 2 else ny
    for p, s in enumerate(parts):
        first, count = slabs.part_range(n, 3, p)
        grid = U.reshape(nz, ny, nx, 5)
        ref = grid[first:first + count] if ax == 2 else grid[:, first:first + count]
        assert np.array_equal(s, ref.reshape(-1, 5))
    assert np.array_equal(slabs.join_states(params, parts), U)
