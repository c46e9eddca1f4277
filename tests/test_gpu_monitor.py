"""The monitor (fvg_monitor) against the reference's: the volume averages of its monitor file (mass, kinetic energy,
total energy; Simulation::volume_averages, cpp/src/SimulationRun.cpp:44-64) of every step of a Taylor-Green run of the
plain FP64 form bit for bit against the reference run alongside on the host (the reference compiled from its sources,
oracle/_ref), and the enstrophy against the oracle's restatement of the reference's validation-script definition."""
import math

import numpy as np
import pytest

import cases
from fenice_b200 import Run
from oracle.oracle import Reference, enstrophy, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="the reference is not compiled (oracle/_ref)")]


def tgv_params(n):
    L = 2 * math.pi
    return dict(nx=n, ny=n, nz=n, Lx=L, Ly=L, Lz=L, gamma=1.4, use_viscous=True, mu=6.25e-4, pr=0.71, reconstruction="weno5",
                riemann_solver="lowmach", time_scheme="SSP Runge-Kutta 3", cfl=0.5, **cases.bcs("periodic", "periodic", "periodic", "periodic"))


def bits(x):
    return np.asarray(x, dtype=np.float64).view(np.uint64)


def test_kinetic_energy_history_of_the_plain_form_is_the_reference_s():
    """48^3 Taylor-Green (the C2 settings), 25 steps from the reference's own initial profile: the monitor's three
    volume averages after every step, in the reference's summation order, have the reference's bits."""
    n, steps = 48, 25
    params = tgv_params(n)
    ref = Reference(params, initial_profile="taylor_green_3d")
    run = Run(params, U=ref.state(), precision=0)
    ke = []
    for k in range(steps + 1):
        got = run.monitor("reference")
        want = ref.volume_averages()
        assert np.array_equal(bits([got["mass"], got["kinetic_energy"], got["total_energy"]]), bits(want)), (k, got, want)
        ke.append(got["kinetic_energy"])
        if k < steps:
            assert run.run(1e30, max_steps=1) == 1
            assert len(ref.steps(1, 1e30)[0]) == 1
    print(f"\nkinetic energy {ke[0]:.15e} -> {ke[-1]:.15e} over {steps} steps, every step the reference's bits")
    assert ke[-1] < ke[0]   # viscous decay


@pytest.mark.parametrize("name,params,seed", [
    ("tgv3d_40_periodic", tgv_params(40), None),
    ("box3d_walls", dict(nx=20, ny=18, nz=16, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3",
                         **cases.bcs("wall", "transmissive", "periodic", "periodic", z=("wall", "outlet"))), 5),
    ("box2d_mixed_sides", dict(nx=48, ny=40, reconstruction="muscl", time_scheme="SSP Runge-Kutta 2",
                               **cases.bcs("periodic", "periodic", "wall", "transmissive")), 6),
], ids=lambda v: v if isinstance(v, str) else "")
def test_enstrophy_and_fast_order(name, params, seed):
    """The enstrophy against the oracle (central differences, wrapped or one-sided), and the fast summation order within
    rounding of the reference's."""
    import bench

    U0 = bench.tgv_state(params["nx"]) if seed is None else cases.case_field(params, seed)
    run = Run(params, U=U0, precision=0)
    run.run(1e30, max_steps=3)
    U = run.state()
    p = run.params
    want = enstrophy(U, (p["nx"], p["ny"], p["nz"]), (p["Lx"], p["Ly"], p["Lz"]),
                     [p[f"bc_{a}min"] == "periodic" and p[f"bc_{a}max"] == "periodic" for a in "xyz"])
    ref_order, fast = run.monitor("reference"), run.monitor("fast")
    print(f"\n{name}: enstrophy {fast['enstrophy']:.15e} (oracle {want:.15e}); kinetic energy {ref_order['kinetic_energy']:.15e} "
          f"(fast order {fast['kinetic_energy']:.15e})")
    assert abs(fast["enstrophy"] - want) <= 1e-12 * abs(want)
    assert ref_order["enstrophy"] == fast["enstrophy"]
    for k in ("mass", "kinetic_energy", "total_energy"):
        assert abs(fast[k] - ref_order[k]) <= 1e-13 * abs(ref_order[k])
