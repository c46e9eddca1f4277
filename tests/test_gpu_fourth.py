"""flux_quadrature = fourth on the device against the reference (tests/golden/fourth.npz, written by
tests/golden/make_fourth.py from the reference compiled from its sources): the residual and its wave speed, and runs of
the reference's time loop, bit for bit (WENO3-Z / WENO5-Z of the conserved averages with the admissibility fallback,
point values and the transverse flux correction where the faces around are smooth, second order at shocks and beside
sides without ghost layers; periodic axes, walls, inlets, outlets, a non-reflecting outlet, the stiffened gas, the
viscous term, the body force)."""
import json
import os

import numpy as np
import pytest

import regression_cases as rc
from fenice_b200 import Run

pytestmark = pytest.mark.gpu

FX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fourth.npz"))
NAMES = sorted({k.split("/")[0] for k in FX.files if k.endswith("/params")})


def nvar(p):
    return 5 if int(p.get("nz", 1)) > 1 else 4


@pytest.mark.parametrize("name", NAMES)
def test_residual_matches_the_reference(name):
    p = json.loads(str(FX[f"{name}/params"]))
    run = Run(p, U=FX[f"{name}/U0"])
    try:
        R, s = run.residual()
        nv = nvar(p)
        assert rc.bits_equal(R[:, :nv], FX[f"{name}/R"][:, :nv]), rc.rel_diff(R[:, :nv], FX[f"{name}/R"][:, :nv])
        assert s == float(FX[f"{name}/s"])
    finally:
        run.close()


@pytest.mark.parametrize("name", NAMES)
def test_time_loop_matches_the_reference(name):
    p = json.loads(str(FX[f"{name}/params"]))
    dts = FX[f"{name}/dts"]
    run = Run(p, U=FX[f"{name}/U0"])
    try:
        assert run.run(float(p["t_end"]), max_steps=len(dts)) == len(dts)
        nv = nvar(p)
        U = run.state()
        assert rc.bits_equal(U[:, :nv], FX[f"{name}/U"][:, :nv]), rc.rel_diff(U[:, :nv], FX[f"{name}/U"][:, :nv])
        assert run.t == float(FX[f"{name}/t"])
    finally:
        run.close()
