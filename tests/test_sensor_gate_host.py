"""The oracle of the learned sensor's gate (oracle/sensor_oracle.py gate_tiles) on hand-worked cases, without a GPU:
the dilation wraps across periodic sides and stops at the others, the tile is extended by one cell along the sweep axis,
and a tile whose extension leaves the mesh across a side that is not periodic stays WENO5-Z."""
import numpy as np

from oracle.sensor_oracle import gate_tiles


def test_one_flagged_cell_2d():
    f = np.zeros((2, 1, 20, 30), np.uint8)
    f[0, 0, 5, 7] = 1   # (x 7, y 5), flagged along x
    g = gate_tiles(f, (16, 15, 1), 2, (True, False, False))
    # x sweeps: only the tile holding x 5..9, y 3..7; y sweeps: every tile touches a side along y that is not periodic
    assert g[0].ravel().tolist() == [1, 0, 0, 0]
    assert g[1].ravel().tolist() == [1, 1, 1, 1]


def test_dilation_wraps_only_across_periodic_sides():
    f = np.zeros((2, 1, 30, 32), np.uint8)
    f[0, 0, 20, 31] = 1   # the last column
    per = gate_tiles(f, (16, 15, 1), 1, (True, True, False))
    # x periodic: the column's neighbour x = 0 lies in the first tile column (and its extension wraps too)
    assert per[0, 0, 1, 0] == 1 and per[0, 0, 1, 1] == 1 and per[0, 0, 0].sum() == 0
    bounded = gate_tiles(f, (16, 15, 1), 1, (False, True, False))
    # x bounded: every x sweep tile touches an x side (its extension leaves the mesh), so all stay WENO5-Z
    assert bounded[0].all()
    # y sweeps, y periodic, the flag is along x only: nothing flagged along y
    assert per[1].sum() == 0 and bounded[1].sum() == 0


def test_radius_reaches_the_neighbouring_tile_3d():
    f = np.zeros((3, 16, 16, 16), np.uint8)
    f[2, 4, 4, 4] = 1   # flagged along z at (4, 4, 4)
    per = (True, True, True)
    g = gate_tiles(f, (8, 8, 8), 3, per)
    # the box 1..7 per axis: x and y stay in tile 0; along z (the sweep axis) the tile above, extended down to z 7, sees it
    assert g[2, 0, 0, 0] == 1 and g[2, 1, 0, 0] == 1 and g[2].sum() == 2 and g[0].sum() == 0 and g[1].sum() == 0
    # radius 4: the box 0..8 reaches the second tile along every axis
    assert gate_tiles(f, (8, 8, 8), 4, per)[2].sum() == 8
    # a flag at 1 with radius 2: the box -1..3 wraps to 15 on a periodic mesh (the second tile again), stops at 0 otherwise
    f2 = np.zeros_like(f)
    f2[2, 1, 1, 1] = 1
    assert gate_tiles(f2, (8, 8, 8), 2, per)[2].sum() == 8 and gate_tiles(f2, (8, 8, 8), 2, (False, False, False))[2, 0, 0, 0] == 1
