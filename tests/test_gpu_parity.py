"""Parity of the CUDA path with the reference, through the C ABI, on a B200.

Plain form (FP64): bit for bit. Every residual, dt, wave speed and state is compared as raw 64-bit patterns with the
golden fixtures the reference wrote (tests/golden/make_golden.py) and, at larger sizes, with the C restatement of the
reference (oracle/fv_oracle.c), which the CPU tests pin to the reference itself."""
import json
import os

import numpy as np
import pytest

import cases
from fenice_b200 import Run
from oracle.oracle import Oracle, fingerprint

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a, dtype=np.float64).view(np.uint64), np.ascontiguousarray(b, dtype=np.float64).view(np.uint64))


def describe(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return f"max |diff| {d.max():.3e}, {int((np.asarray(a).view(np.uint64) != np.asarray(b).view(np.uint64)).sum())} values differ"


@pytest.mark.parametrize("case", cases.RESIDUAL_CASES, ids=[c[0] for c in cases.RESIDUAL_CASES])
def test_residual_bit_exact(golden, case):
    name = case[0]
    g = golden[0]
    params = json.loads(str(g[f"{name}/params"]))
    run = Run(params, U=g[f"{name}/U"])
    R, s = run.residual(predictor_half_dt=float(g[f"{name}/half_dt"]))
    assert bits_equal(R, g[f"{name}/R"]), describe(R, g[f"{name}/R"])
    assert s == float(g[f"{name}/smax"])
    # the state is untouched by a residual
    assert bits_equal(run.state(), g[f"{name}/U"])


@pytest.mark.parametrize("case", cases.STEP_CASES, ids=[c[0] for c in cases.STEP_CASES])
def test_steps_bit_exact(golden, case):
    name, _, _, n = case
    g = golden[1]
    params = json.loads(str(g[f"{name}/params"]))
    run = Run(params, U=g[f"{name}/U0"])
    dts, sms = [], []
    for _ in range(n):
        r = run.step(1e30)
        dts.append(r.dt)
        sms.append(r.s_max)
    assert bits_equal(dts, g[f"{name}/dts"]), (dts, g[f"{name}/dts"])
    assert bits_equal(sms, g[f"{name}/smaxs"])
    assert bits_equal(run.state(), g[f"{name}/U"]), describe(run.state(), g[f"{name}/U"])
    assert run.t == float(g[f"{name}/t"])


@pytest.mark.parametrize("case", cases.STEP_CASES, ids=[c[0] for c in cases.STEP_CASES])
def test_graph_run_bit_exact(golden, case):
    """The same steps through fvg_run_until (CUDA graphs, clock on the device), stopping on the step limit."""
    name, _, _, n = case
    g = golden[1]
    params = json.loads(str(g[f"{name}/params"]))
    run = Run(params, U=g[f"{name}/U0"])
    assert run.run(1e30, max_steps=n) == n
    assert bits_equal(run.state(), g[f"{name}/U"]), describe(run.state(), g[f"{name}/U"])
    assert run.t == float(g[f"{name}/t"])


def test_run_stops_at_t_end(golden):
    """t_end clamps the last dt (dt = min(dt, t_end - t)) and the loop ends at t_end, as the reference's loop."""
    name = "hancock_vl_2d"
    g = golden[1]
    params = json.loads(str(g[f"{name}/params"]))
    t_end = float(g[f"{name}/t"])
    run = Run(params, U=g[f"{name}/U0"])
    steps = run.run(t_end)
    assert steps == 5 and run.t == t_end
    assert bits_equal(run.state(), g[f"{name}/U"])
    orc = Oracle()
    U, t, dts, _, _ = orc.run(params, g[f"{name}/U0"], 100, t_end=0.75 * t_end)
    run2 = Run(params, U=g[f"{name}/U0"])
    assert run2.run(0.75 * t_end) == len(dts)
    assert bits_equal(run2.state(), U) and run2.t == t


@pytest.mark.parametrize("eos_kind", [0, 1])
@pytest.mark.parametrize("riemann", [0, 1])
def test_riemann_fingerprint(eos_kind, riemann):
    """The reference's bench_riemann hash over its 65536 state pairs (edge cases included), on the device."""
    with open(os.path.join(HERE, "golden", "riemann.json")) as f:
        hashes = json.load(f)["hashes"]
    key = ("ideal" if eos_kind == 0 else "stiffened") + " " + ("HLLC" if riemann == 0 else "Low-Mach")
    UL, UR, ax = Oracle().riemann_pool(eos_kind)
    params = dict(nx=4, ny=4, shock_blend=0.0, riemann_solver=["HLLC", "lowmach"][riemann],
                  eos_type=["Ideal Gas", "Stiffened Gas"][eos_kind], gamma=[1.4, 4.4][eos_kind], p_inf=[0.0, 6.0e8][eos_kind])
    F, S = Run(params).face_flux_batch(UL, UR, ax)
    assert f"{fingerprint(F, S):016x}" == hashes[key]


def test_state_round_trip_and_2d_rho_w():
    U = cases.smooth_field(37, 23, seed=3)
    run = Run(dict(nx=37, ny=23), U=U)
    assert bits_equal(run.state(), U)
    bad = U.copy()
    bad[5, 4] = 1.0
    with pytest.raises(ValueError):
        run.set_state(bad)


@pytest.mark.parametrize("params,seed,n", [
    (dict(nx=40, ny=36, nz=34, reconstruction="weno5", riemann_solver="lowmach", time_scheme="SSP Runge-Kutta 3", use_viscous=True,
          mu=6.25e-4, pr=0.71, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, **cases.bcs("periodic", "periodic", "periodic", "periodic")), 31, 2),
    (dict(nx=130, ny=97, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4, **cases.bcs("transmissive", "transmissive",
          "transmissive", "transmissive")), 32, 3),
    (dict(nx=96, ny=80, Lx=8.0, Ly=12.0, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock", u_in=2.0, rho_in=1.4,
          p_out=1.0, **cases.bcs("vel_inlet", "transmissive", "transmissive", "transmissive")), 33, 6),
])
def test_larger_meshes_vs_oracle(params, seed, n):
    """Meshes of many tiles (partial tiles at the edges) against the restatement."""
    U0 = cases.case_field(params, seed)
    U, t, dts, sms, _ = Oracle().run(params, U0, n)
    run = Run(params, U=U0)
    assert run.run(1e30, max_steps=n) == n
    assert bits_equal(run.state(), U), describe(run.state(), U)
    assert run.t == t
