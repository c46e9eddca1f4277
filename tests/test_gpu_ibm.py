"""The immersed body (sharp ghost-cell wall) on the GPU against the reference, bit for bit: fixtures the reference wrote
(tests/golden/ibm.npz: a residual of a forced perturbed state, then a few steps, for a 2-D cylinder with MUSCL-Hancock,
WENO5-Z / SSP-RK3 (the narrow stencil beside the body) and boundary_order 1, a 3-D sphere, and a 3-D cylinder with viscous
no-slip walls), and a longer Mach 2 cylinder run against the reference run alongside (when oracle/_ref is built)."""
import json
import math
import os

import numpy as np
import pytest

import cases
from fenice_b200 import Run
from oracle.oracle import Reference, ref_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ibm_golden():
    import os

    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ibm.npz"))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def describe(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return f"max |diff| {d.max():.3e} at {np.unravel_index(d.argmax(), d.shape)}, {int((d > 0).sum())} values differ"


@pytest.mark.parametrize("case", cases.IBM_CASES, ids=[c[0] for c in cases.IBM_CASES])
def test_ibm_residual_bit_exact(ibm_golden, case):
    name = case[0]
    g = ibm_golden
    params = json.loads(str(g[f"{name}/params"]))
    run = Run(params, U=g[f"{name}/U0"])
    R, s = run.residual(predictor_half_dt=float(g[f"{name}/half_dt"]))
    assert bits_equal(R, g[f"{name}/R"]), describe(R, g[f"{name}/R"])
    assert s == float(g[f"{name}/smax"])


@pytest.mark.parametrize("case", cases.IBM_CASES, ids=[c[0] for c in cases.IBM_CASES])
def test_ibm_steps_bit_exact(ibm_golden, case):
    name, _, _, _, n = case
    g = ibm_golden
    params = json.loads(str(g[f"{name}/params"]))
    run = Run(params, U=g[f"{name}/U0"])
    assert run.run(1e30, max_steps=n) == n
    assert bits_equal(run.state(), g[f"{name}/U"]), describe(run.state(), g[f"{name}/U"])
    assert run.t == float(g[f"{name}/t"])


def test_ibm_mixed_form_within_bar(ibm_golden):
    name = "cyl_weno5_rk3"
    g = ibm_golden
    params = json.loads(str(g[f"{name}/params"]))
    plain = Run(params, U=g[f"{name}/U0"], precision=0)
    mixed = Run(params, U=g[f"{name}/U0"], precision=1)
    plain.run(1e30, max_steps=20)
    mixed.run(1e30, max_steps=20)
    Up, Um = plain.state(), mixed.state()
    l1 = np.abs(Um[:, 0] - Up[:, 0]).sum() / np.abs(Up[:, 0]).sum()
    print(f"\ncylinder WENO5 mixed vs FP64, 20 steps: L1 rho {l1:.2e}")
    assert l1 <= 1e-4


@pytest.mark.skipif(not ref_available(), reason="the reference is not compiled (oracle/_ref)")
def test_mach2_cylinder_against_reference():
    """Configuration C5 at a quarter of its resolution (400 x 600), from the free stream, 150 MUSCL-Hancock (MC) steps."""
    c = math.sqrt(1.4 * 1.0 / 1.4)
    params = dict(nx=400, ny=600, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock", riemann_solver="HLLC",
                  cfl=0.5, **dict(cases.CYL, u_in=2.0 * c))
    ref = Reference(params, initial_state=(1.4, 2.0 * c, 0.0, 1.0))
    run = Run(params, U=ref.state())
    assert run.run(1e30, max_steps=150) == 150
    ref.steps(150, 1e30)
    assert bits_equal(run.state(), ref.state()), describe(run.state(), ref.state())
    assert run.t == ref.t
    # the monitor's loads (Simulation::ibm_loads of a residual of the state): the same sums in the same order
    loads, ref_loads = run.ibm_loads(), ref.ibm_loads()
    print(f"\nloads after 150 steps: {loads}")
    assert [loads["Fx"], loads["Fy"], loads["Mz"]] == ref_loads


def test_sensor_gate_with_the_immersed_body():
    """The learned gate on a mixed WENO5-Z cylinder run: the narrow stencil beside the body keeps its WENO3-Z; a gate
    that never passes a tile gives the plain mixed run's state."""
    from fenice_b200 import diagnostics as D
    from fenice_b200.sensor import Sensor

    params = D.cylinder_params(160, 240, form="mixed")
    U0 = D.free_stream(params)
    plain = Run(params, U=U0, precision=1)
    plain.run(1e30, max_steps=30)
    s = Sensor.load(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "fenice_b200", "sensor_weights.npz"))
    never = Run(params, U=U0, precision=1)
    never.set_sensor(s, -1e30)
    never.run(1e30, max_steps=30)
    assert np.abs(never.state() - plain.state()).max() <= 1e-5 * np.abs(plain.state()).max()
    gated = Run(params, U=U0, precision=1)
    gated.set_sensor(s, float(s.meta["threshold"]))
    gated.run(1e30, max_steps=30)
    lin, ev = gated.sensor_counts()
    l1 = np.abs(gated.state()[:, 0] - plain.state()[:, 0]).sum() / np.abs(plain.state()[:, 0]).sum()
    print(f"\ncylinder, sensor gate: {lin}/{ev} tile-axes linear, L1(rho) vs plain mixed {l1:.2e}")
    assert ev > 0 and l1 < 1e-2
