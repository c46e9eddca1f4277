"""Case-file source terms and time-dependent boundary values on the device against the reference
(tests/golden/sources.npz, written by tests/golden/make_sources.py from the reference compiled from its sources):
residuals at given stage times (fvg_set_stage_time; the MUSCL-Hancock predictor's too) and whole runs of its time loop.

Steady sources (evaluated once on the host with the C library's functions, as the reference) and boundary values from
time tables or arithmetic expressions of t give the reference's bits. Sources that read t, and boundary values with
transcendental functions of t, are evaluated on the device at every stage with CUDA's functions: there the states are
within 1e-12 (relative, per variable) of the reference's. A boundary value that stops being positive stops the run with
an error, as the reference's does. A slab-decomposed run reproduces the whole run's bits."""
import json
import os
import re

import numpy as np
import pytest

import regression_cases as rc
from fenice_b200 import Run
from fenice_b200.slabs import run_decomposed

pytestmark = pytest.mark.gpu

FX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sources.npz"))
NAMES = sorted({k.split("/")[0] for k in FX.files if k.endswith("/params")})
EXACT = {"steady_weno5_rk3_3d", "steady_hancock_bodyforce_2d", "table_inlet_outlet_rk2_2d", "expr_massflow_weno3_2d"}
DEVICE_MATH = {"unsteady_muscl_rk3_2d", "unsteady_hancock_3d", "expr_moving_wall_viscous_2d"}
TOL = 1e-12


def params_of(name, tmp_path):
    p = json.loads(str(FX[f"{name}/params"]))
    for k, v in list(p.items()):
        if k.endswith("_table"):
            path = tmp_path / v
            path.write_text(str(FX[f"table/{v}"]))
            p[k] = str(path)
    return p


def nvar(p):
    return 5 if int(p.get("nz", 1)) > 1 else 4


def check(name, got, want, what):
    got, want = np.asarray(got)[:, : want.shape[1]], np.asarray(want)
    if name in EXACT:
        assert rc.bits_equal(got, want), f"{what}: relative difference {rc.rel_diff(got, want):.3g}"
    else:
        assert rc.rel_diff(got, want) < TOL, f"{what}: relative difference {rc.rel_diff(got, want):.3g}"


def test_fixture_cases_are_classified():
    assert set(NAMES) == EXACT | DEVICE_MATH | {"falling_p_out_rk3_2d"}


@pytest.mark.parametrize("name", sorted(EXACT | DEVICE_MATH))
def test_residual_at_stage_times_matches_the_reference(name, tmp_path):
    p = params_of(name, tmp_path)
    nv = nvar(p)
    run = Run(p, U=FX[f"{name}/U0"])
    try:
        hancock = p["time_scheme"] == "MUSCL-Hancock"
        for i, st in enumerate(FX[f"{name}/stage_times"]):
            run.set_stage_time(float(st))
            R, s = run.residual()
            check(name, R[:, :nv], FX[f"{name}/R{i}"][:, :nv], f"residual at t = {st}")
            assert s == float(FX[f"{name}/s{i}"]) or (name in DEVICE_MATH and abs(s / float(FX[f"{name}/s{i}"]) - 1) < TOL)
            if hancock:
                run.set_stage_time(float(st) + 0.004)
                Rh, sh = run.residual(predictor_half_dt=0.004)
                check(name, Rh[:, :nv], FX[f"{name}/Rh{i}"][:, :nv], f"predictor residual at t = {st + 0.004}")
        run.set_stage_time()
    finally:
        run.close()


@pytest.mark.parametrize("name", sorted(EXACT | DEVICE_MATH))
def test_time_loop_matches_the_reference(name, tmp_path):
    p = params_of(name, tmp_path)
    dts = FX[f"{name}/dts"]
    run = Run(p, U=FX[f"{name}/U0"])
    try:
        steps = run.run(float(p["t_end"]), max_steps=len(dts))
        assert steps == len(dts)
        U = run.state()
        check(name, U[:, : nvar(p)], FX[f"{name}/U"][:, : nvar(p)], "state")
        if name in EXACT:
            assert run.t == float(FX[f"{name}/t"])
        else:
            assert abs(run.t - float(FX[f"{name}/t"])) <= TOL * float(FX[f"{name}/t"])
    finally:
        run.close()


def test_a_boundary_value_that_stops_being_positive_stops_the_run(tmp_path):
    name = "falling_p_out_rk3_2d"
    p = params_of(name, tmp_path)
    at = float(re.search(r"at t=([0-9.eE+-]+)", str(FX[f"{name}/error"])).group(1))   # the reference's stage time
    run = Run(p, U=FX[f"{name}/U0"])
    try:
        with pytest.raises(RuntimeError, match="p_out") as e:
            run.run(1.0, max_steps=200)
        ours = float(re.search(r"at t = ([0-9.eE+-]+)", str(e.value)).group(1))
        assert abs(ours - at) < 1e-6   # (the reference prints the time with 6 decimals)
    finally:
        run.close()


@pytest.mark.parametrize("name", ["unsteady_muscl_rk3_2d", "unsteady_hancock_3d", "table_inlet_outlet_rk2_2d", "steady_weno5_rk3_3d"])
def test_decomposed_run_equals_the_whole_run(name, tmp_path):
    p = params_of(name, tmp_path)
    n = len(FX[f"{name}/dts"])
    whole = Run(p, U=FX[f"{name}/U0"])
    try:
        whole.run(float(p["t_end"]), max_steps=n)
        W = whole.state()
    finally:
        whole.close()
    U, steps, t = run_decomposed(p, FX[f"{name}/U0"], 2, float(p["t_end"]), max_steps=n)
    assert steps == n
    assert rc.bits_equal(U, W)
