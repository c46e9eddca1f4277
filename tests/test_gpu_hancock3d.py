"""3-D MUSCL-Hancock on the GPU against the reference, bit for bit (fixtures tests/golden/hancock3d.npz, written by the
reference's MusclReconstruction::hancock_residual_3d through tests/golden/make_golden.py): residuals with the predictor of
half a step and steps of the MUSCL-Hancock scheme for periodic, slab and first-order sides, walls on every axis, every
limiter and both Riemann solvers; and a mesh of many 8 x 8 x 4 tiles against the restatement (oracle/)."""
import json
import os

import numpy as np
import pytest

import cases
from fenice_b200 import Run
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hancock3d.npz"))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def describe(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return f"max |diff| {d.max():.3e} at {np.unravel_index(d.argmax(), d.shape)}, {int((d > 0).sum())} values differ"


@pytest.mark.parametrize("case", cases.HANCOCK3D_RESIDUAL_CASES, ids=[c[0] for c in cases.HANCOCK3D_RESIDUAL_CASES])
def test_hancock3d_residual_bit_exact(fx, case):
    name = case[0]
    run = Run(json.loads(str(fx[f"{name}/params"])), U=fx[f"{name}/U"])
    R, s = run.residual(predictor_half_dt=float(fx[f"{name}/half_dt"]))
    assert bits_equal(R, fx[f"{name}/R"]), describe(R, fx[f"{name}/R"])
    assert s == float(fx[f"{name}/smax"])
    assert bits_equal(run.state(), fx[f"{name}/U"])


@pytest.mark.parametrize("case", cases.HANCOCK3D_STEP_CASES, ids=[c[0] for c in cases.HANCOCK3D_STEP_CASES])
def test_hancock3d_steps_bit_exact(fx, case):
    name, _, _, n = case
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


@pytest.mark.parametrize("case", cases.HANCOCK3D_STEP_CASES, ids=[c[0] for c in cases.HANCOCK3D_STEP_CASES])
def test_hancock3d_graph_run_bit_exact(fx, case):
    """The same steps through fvg_run_until (CUDA graphs of two steps: the predictor's ping-pong)."""
    name, _, _, n = case
    run = Run(json.loads(str(fx[f"{name}/params"])), U=fx[f"{name}/U0"])
    assert run.run(1e30, max_steps=n) == n
    assert bits_equal(run.state(), fx[f"{name}/U"]), describe(run.state(), fx[f"{name}/U"])
    assert run.t == float(fx[f"{name}/t"])


def test_hancock3d_many_tiles_vs_oracle():
    """A mesh of 5 x 4 x 9 tiles (partial at every high side) with an inlet, walls and a periodic axis, against the
    restatement."""
    params = dict(nx=37, ny=30, nz=33, Lx=2.0, Ly=1.6, Lz=1.8, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock",
                  u_in=1.2, rho_in=1.3, p_out=1.0, **cases.bcs("vel_inlet", "transmissive", "wall", "no_slip", z=("periodic", "periodic")))
    U0 = cases.case_field(params, 39)
    U, t, dts, sms, _ = Oracle().run(params, U0, 4)
    run = Run(params, U=U0)
    assert run.run(1e30, max_steps=4) == 4
    assert bits_equal(run.state(), U), describe(run.state(), U)
    assert run.t == t
