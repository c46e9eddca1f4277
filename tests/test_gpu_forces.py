"""The body force (ConstantBodyForce, cpp/src/Physics.cpp:832-844) and MUSCL-Hancock with viscous fluxes on the GPU
against the reference, bit for bit (fixtures tests/golden/forces.npz, written by the reference through
tests/golden/make_golden.py): a residual (MUSCL-Hancock: with the predictor of half a step, which the body force joins
and the viscous term does not) and steps, 2-D and 3-D, every time scheme; and the combinations the device refuses."""
import json
import os

import numpy as np
import pytest

import cases
from fenice_b200 import Run

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "forces.npz"))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def describe(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return f"max |diff| {d.max():.3e} at {np.unravel_index(d.argmax(), d.shape)}, {int((d > 0).sum())} values differ"


@pytest.mark.parametrize("case", cases.FORCE_CASES, ids=[c[0] for c in cases.FORCE_CASES])
def test_force_residual_bit_exact(fx, case):
    name = case[0]
    run = Run(json.loads(str(fx[f"{name}/params"])), U=fx[f"{name}/U0"])
    R, s = run.residual(predictor_half_dt=float(fx[f"{name}/half_dt"]))
    assert bits_equal(R, fx[f"{name}/R"]), describe(R, fx[f"{name}/R"])
    assert s == float(fx[f"{name}/smax"])


@pytest.mark.parametrize("case", cases.FORCE_CASES, ids=[c[0] for c in cases.FORCE_CASES])
def test_force_steps_bit_exact(fx, case):
    name, n = case[0], case[4]
    run = Run(json.loads(str(fx[f"{name}/params"])), U=fx[f"{name}/U0"])
    dts, sms = [], []
    for _ in range(n):
        r = run.step(1e30)
        dts.append(r.dt)
        sms.append(r.s_max)
    assert bits_equal(dts, fx[f"{name}/dts"]), (dts, fx[f"{name}/dts"])
    assert bits_equal(sms, fx[f"{name}/smaxs"])
    assert bits_equal(run.state(), fx[f"{name}/U"]), describe(run.state(), fx[f"{name}/U"])
    assert run.t == float(fx[f"{name}/t"])


@pytest.mark.parametrize("case", cases.FORCE_CASES, ids=[c[0] for c in cases.FORCE_CASES])
def test_force_graph_run_bit_exact(fx, case):
    name, n = case[0], case[4]
    run = Run(json.loads(str(fx[f"{name}/params"])), U=fx[f"{name}/U0"])
    assert run.run(1e30, max_steps=n) == n
    assert bits_equal(run.state(), fx[f"{name}/U"]), describe(run.state(), fx[f"{name}/U"])


def test_body_force_refusals(fx):
    p = json.loads(str(fx["grav_muscl_rk2_2d/params"]))
    U = fx["grav_muscl_rk2_2d/U0"]
    with pytest.raises(ValueError, match="FP64 form only"):
        Run(p, U=U, precision=1)
