"""The cell engine's host side without a GPU: the leaf order of fenice_b200.cells.base_leaves against the reference's own
CellMesh (its sort by level and Morton key, oracle/_ref), and the configurations and leaf lists fvg_cells_create refuses
before it touches a device."""
import numpy as np
import pytest

from fenice_b200.cells import CellEngine, base_leaves
from oracle.oracle import Reference, ReferenceCells, ref_available

P3 = dict(nx=9, ny=7, nz=5, Lx=1.7, Ly=1.1, Lz=0.9, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3",
          bc_xmin="wall", bc_xmax="outlet", bc_ymin="periodic", bc_ymax="periodic", bc_zmin="transmissive", bc_zmax="wall")
P2 = dict(nx=13, ny=6, reconstruction="muscl", bc_xmin="periodic", bc_xmax="periodic", bc_ymin="wall", bc_ymax="wall")


@pytest.mark.skipif(not ref_available(), reason="the reference is not compiled (oracle/_ref)")
@pytest.mark.parametrize("params", [P3, P2], ids=["3d", "2d"])
def test_morton_order_is_the_reference_cellmesh_order(params):
    rc = ReferenceCells(Reference(params, initial_state=(1, 0, 0, 1, 0)), 2)
    lv, ci, cj, ck = base_leaves(params)
    assert np.array_equal(rc.level, lv) and np.array_equal(rc.ci, ci) and np.array_equal(rc.cj, cj) and np.array_equal(rc.ck, ck)


def refused(params, lv, ci, cj, ck, match):
    with pytest.raises(ValueError, match=match):
        CellEngine(params, lv, ci, cj, ck)


def test_refusals():
    lv, ci, cj, ck = base_leaves(P3)
    bad = lv.copy()
    bad[7] = 1
    refused(P3, bad, ci, cj, ck, "only level-0 leaves")
    dup = ci.copy()
    dup[3] = ci[4]
    dup_j, dup_k = cj.copy(), ck.copy()
    dup_j[3], dup_k[3] = cj[4], ck[4]
    refused(P3, lv, dup, dup_j, dup_k, "are the same cell")
    refused(P3, lv[:-1], ci[:-1], cj[:-1], ck[:-1], "do not tile")
    out = ci.copy()
    out[0] = 9
    refused(P3, lv, out, cj, ck, "outside the base mesh")
    for extra, what in ((dict(bc_xmax="non_reflecting"), "non-reflecting"), (dict(positivity_fallback=True), "positivity_fallback"),
                        (dict(flux_quadrature="fourth"), "fourth")):
        refused(dict(P3, **extra), lv, ci, cj, ck, what)
