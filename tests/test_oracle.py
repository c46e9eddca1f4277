"""The C restatement (oracle/) against the reference: its golden fixtures, its Riemann fingerprints, and, where the
reference compiled from its sources is present (oracle/_ref), the reference itself on further seeded inputs."""
import json
import os

import numpy as np
import pytest

import cases
from oracle.oracle import Oracle, Reference, ref_available

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def orc():
    return Oracle()


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


@pytest.mark.parametrize("case", cases.RESIDUAL_CASES, ids=[c[0] for c in cases.RESIDUAL_CASES])
def test_oracle_residual_matches_golden(orc, golden, case):
    name = case[0]
    g = golden[0]
    params = json.loads(str(g[f"{name}/params"]))
    R, s = orc.residual(params, g[f"{name}/U"], float(g[f"{name}/half_dt"]))
    assert bits_equal(R, g[f"{name}/R"]), np.abs(R - g[f"{name}/R"]).max()
    assert s == float(g[f"{name}/smax"])


@pytest.mark.parametrize("case", cases.STEP_CASES, ids=[c[0] for c in cases.STEP_CASES])
def test_oracle_steps_match_golden(orc, golden, case):
    name, _, _, n = case
    g = golden[1]
    params = json.loads(str(g[f"{name}/params"]))
    U, t, dts, sms, _ = orc.run(params, g[f"{name}/U0"], n)
    assert bits_equal(dts, g[f"{name}/dts"])
    assert bits_equal(sms, g[f"{name}/smaxs"])
    assert bits_equal(U, g[f"{name}/U"])
    assert t == float(g[f"{name}/t"])


@pytest.fixture(scope="module")
def h3():
    return np.load(os.path.join(HERE, "golden", "hancock3d.npz"))


@pytest.mark.parametrize("case", cases.HANCOCK3D_RESIDUAL_CASES, ids=[c[0] for c in cases.HANCOCK3D_RESIDUAL_CASES])
def test_oracle_hancock3d_residual_matches_golden(orc, h3, case):
    name = case[0]
    params = json.loads(str(h3[f"{name}/params"]))
    R, s = orc.residual(params, h3[f"{name}/U"], float(h3[f"{name}/half_dt"]))
    assert bits_equal(R, h3[f"{name}/R"]), np.abs(R - h3[f"{name}/R"]).max()
    assert s == float(h3[f"{name}/smax"])


@pytest.mark.parametrize("case", cases.HANCOCK3D_STEP_CASES, ids=[c[0] for c in cases.HANCOCK3D_STEP_CASES])
def test_oracle_hancock3d_steps_match_golden(orc, h3, case):
    name, _, _, n = case
    params = json.loads(str(h3[f"{name}/params"]))
    U, t, dts, sms, _ = orc.run(params, h3[f"{name}/U0"], n)
    assert bits_equal(dts, h3[f"{name}/dts"])
    assert bits_equal(U, h3[f"{name}/U"])
    assert t == float(h3[f"{name}/t"])


def test_oracle_riemann_fingerprints(orc):
    with open(os.path.join(HERE, "golden", "riemann.json")) as f:
        h = json.load(f)["hashes"]
    assert f"{orc.riemann_hash(0, 0):016x}" == h["ideal HLLC"]
    assert f"{orc.riemann_hash(0, 1):016x}" == h["ideal Low-Mach"]
    assert f"{orc.riemann_hash(1, 0):016x}" == h["stiffened HLLC"]
    assert f"{orc.riemann_hash(1, 1):016x}" == h["stiffened Low-Mach"]


@pytest.mark.skipif(not ref_available(), reason="the reference is not compiled here (oracle/_ref)")
@pytest.mark.parametrize("seed", [101, 102])
def test_oracle_vs_reference_fresh_inputs(orc, seed):
    """New seeds on a few configurations, restatement vs the compiled reference."""
    for name, params, _, half in cases.RESIDUAL_CASES[::3]:
        U = cases.case_field(params, seed)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        Rr, sr = ref.residual(U, predictor_half_dt=half)
        Ro, so = orc.residual(params, U, half)
        assert bits_equal(Rr, Ro), name
        assert sr == so, name


@pytest.mark.skipif(not ref_available(), reason="the reference is not compiled here (oracle/_ref)")
def test_oracle_vortex_run_vs_reference(orc):
    """The isentropic vortex (the reference's built-in profile) for 20 MUSCL-Hancock steps at 64^2."""
    params = dict(nx=64, ny=64, Lx=10.0, Ly=10.0, reconstruction="muscl", muscl_limiter="Van Leer", riemann_solver="HLLC",
                  time_scheme="MUSCL-Hancock", cfl=0.5, **cases.bcs("periodic", "periodic", "periodic", "periodic"))
    ref = Reference(params, initial_profile="isentropic_vortex")
    U0 = ref.state()
    dts, sms = ref.steps(20, 10.0)
    U, t, odts, osms, _ = orc.run(params, U0, 20, t_end=10.0)
    assert bits_equal(odts, dts) and bits_equal(osms, sms)
    assert bits_equal(U, ref.state())
