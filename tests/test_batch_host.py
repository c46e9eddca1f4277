"""The batched-problem path without a GPU: the host rejects batches the device path does not run before it touches
CUDA, the seeded shock-tube workload is what it says, and the exact Riemann solver of the oracle matches the reference's
own (fixture tests/golden/exact_riemann.npz, written by tests/golden/make_exact.py)."""
import ctypes
import os

import numpy as np
import pytest

from fenice_b200 import initial
from fenice_b200 import params as P
from fenice_b200 import runtime as RT
from oracle.exact_riemann import riemann

HERE = os.path.dirname(os.path.abspath(__file__))


def batch_code(plist):
    lib = RT.load_library()
    cfgs = (P.FvgConfig * max(1, len(plist)))(*[P.to_config(p) for p in plist])
    h = ctypes.c_void_p()
    rc = lib.fvg_batch_create(cfgs, len(plist), ctypes.byref(h))
    return rc, lib.fvg_create_error().decode()


TUBE = dict(nx=128, ny=1, Ly=1 / 128, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", bc_xmin="transmissive", bc_xmax="transmissive",
            bc_ymin="transmissive", bc_ymax="transmissive")


@pytest.mark.parametrize("plist,words", [
    ([], "at least one"),
    ([TUBE, dict(TUBE, reconstruction="muscl")], "share"),
    ([TUBE, dict(TUBE, riemann_solver="HLLC (Low-Mach Thornber)")], "share"),
    ([dict(TUBE, nz=4, bc_zmin="periodic", bc_zmax="periodic")], "2-D"),
    ([dict(TUBE, reconstruction="muscl", time_scheme="MUSCL-Hancock")], "ssp-rk3"),
    ([TUBE, dict(TUBE, nx=0)], "problem 1"),
    ([dict(TUBE, use_ibm=True, ibm_radius=0.1)], "immersed"),
])
def test_batches_the_device_path_does_not_run_are_rejected(plist, words):
    rc, msg = batch_code(plist)
    assert rc == RT.FVG_ERR_CONFIG
    assert words.lower() in msg.lower()


def test_shock_tube_workload():
    params, states, lr = initial.shock_tubes(512, seed=0)
    nx = np.array([p["nx"] for p in params])
    assert len(params) == len(states) == 512
    assert nx.min() >= 128 and nx.max() <= 8192
    # log-uniform: about half the problems below the geometric mean 1024
    assert 0.4 < np.mean(nx < 1024) < 0.6
    for p, U, (left, right) in zip(params, states, lr):
        assert U.shape == (p["nx"], 5) and p["Ly"] == 1.0 / p["nx"]
        for rho, u, pr in (left, right):
            assert 0.1 <= rho <= 1 and -1 <= u <= 1 and 0.05 <= pr <= 1
        assert U[0, 0] == left[0] and U[-1, 0] == right[0]
    again = initial.shock_tubes(512, seed=0)
    assert all(np.array_equal(a, b) for a, b in zip(states, again[1]))


def test_exact_riemann_oracle_matches_the_reference_solver():
    g = np.load(os.path.join(HERE, "golden", "exact_riemann.npz"))
    for k in range(len(g["left"])):
        sol = np.array(riemann(g["x"], float(g["t"]), tuple(g["left"][k]), tuple(g["right"][k])))
        np.testing.assert_allclose(sol, g["solution"][k], rtol=1e-14, atol=1e-15)
