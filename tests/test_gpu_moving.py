"""An immersed body in prescribed motion on the device against the reference's own time loop (tests/golden/moving.npz,
written by tests/golden/make_moving.py with the reference's command-line solver): a translating circle, a circle that
spins within a time window (viscous, no-slip), a translating and turning circle under MUSCL-Hancock, and translating and
spinning spheres (WENO5-Z and viscous MUSCL), and bodies driven by the flow (free, on springs and dampers, spinning, with the centre of mass off the pivot; a free sphere) and bodies under gravity (hydrostatic ghost pressures, loads net
of the weight, a falling circle and sphere) and airfoil sections (NACA 4-digit and a coordinate file: static, pitching,
free to heave and pitch, extruded in 3-D), bit for bit after their steps: the geometry rebuilt every quarter cell, the
cells the body left filled from the wall layer, the ghost and deep cells at the wall's velocity. A body that travels more
than a cell in a step stops the run, as the reference's."""
import json
import os

import numpy as np
import pytest

import regression_cases as rc
from fenice_b200 import Run

pytestmark = pytest.mark.gpu

FX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "moving.npz"))
NAMES = sorted({k.split("/")[0] for k in FX.files if k.endswith("/params")})


def params_of(name, tmp_path):
    p = json.loads(str(FX[f"{name}/params"]))
    if p.get("ibm_file") == "@section.dat":   # a section read from a coordinate file
        (tmp_path / "section.dat").write_text(str(FX["file/section.dat"]))
        p["ibm_file"] = str(tmp_path / "section.dat")
    return p


@pytest.mark.parametrize("name", [n for n in NAMES if f"{n}/error" not in FX.files])
def test_moving_body_run_matches_the_reference(name, tmp_path):
    p = params_of(name, tmp_path)
    n = int(FX[f"{name}/steps"])
    run = Run(p, U=FX[f"{name}/U0"])
    try:
        assert run.run(float(p["t_end"]), max_steps=n) == int(FX[f"{name}/step"])
        U = run.state()
        ref = FX[f"{name}/U"]
        assert rc.bits_equal(U[:, : ref.shape[1]], ref), rc.rel_diff(U, ref)
        assert run.t == float(FX[f"{name}/t"])
    finally:
        run.close()


@pytest.mark.parametrize("name", [n for n in NAMES if f"{n}/error" in FX.files])
def test_a_body_that_outruns_its_ghost_table_stops_the_run(name, tmp_path):
    p = params_of(name, tmp_path)
    run = Run(p, U=FX[f"{name}/U0"])
    try:
        with pytest.raises(RuntimeError, match="travelled more than one cell"):
            run.run(float(p["t_end"]), max_steps=int(FX[f"{name}/steps"]))
        assert "travelled more than one cell" in str(FX[f"{name}/error"])
    finally:
        run.close()
