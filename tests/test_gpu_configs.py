"""Whole runs of the benchmark configurations on the GPU against the reference run alongside on the host (the reference
compiled from its sources, oracle/_ref): the final state bit for bit, the step count, and, where the configuration has
one, the exact solution.

* C1: the isentropic vortex, 256^2, MUSCL Van Leer + HLLC + MUSCL-Hancock, CFL 0.5, one period (t = 10).
* C3 (reduced): a seeded four-quadrant Riemann problem, WENO5-Z + HLLC + SSP-RK3, CFL 0.4, transmissive, 192^2 to t = 0.25.
* C2 (reduced): the Taylor-Green vortex 48^3, WENO5-Z + low-Mach HLLC + SSP-RK3, viscous Re 1600, 10 steps.
"""
import math

import numpy as np
import pytest

import cases
from fenice_b200 import Run
from oracle.oracle import Reference, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="the reference is not compiled (oracle/_ref)")]


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def quadrants(n, seed):
    """Four constant states split at (0.5, 0.5), drawn in NE, NW, SW, SE order: rho, p ~ U[0.1, 2], u, v ~ U[-1, 1]."""
    rng = np.random.default_rng(seed)
    st = [(rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.1, 2)) for _ in range(4)]
    c = (np.arange(n) + 0.5) / n
    y, x = np.meshgrid(c, c, indexing="ij")
    x, y = x.ravel(), y.ravel()
    q = np.where(x >= 0.5, np.where(y >= 0.5, 0, 3), np.where(y >= 0.5, 1, 2))
    W = np.zeros((n * n, 5))
    for k, (r, u, v, p) in enumerate(st):
        W[q == k] = (r, u, v, p, 0.0)
    return cases.prim_to_cons(W)


def test_c1_isentropic_vortex_one_period():
    params = dict(nx=256, ny=256, Lx=10.0, Ly=10.0, gamma=1.4, reconstruction="muscl", muscl_limiter="Van Leer", riemann_solver="HLLC",
                  time_scheme="MUSCL-Hancock", cfl=0.5, **cases.bcs("periodic", "periodic", "periodic", "periodic"))
    ref = Reference(params, initial_profile="isentropic_vortex")
    U0 = ref.state()
    run = Run(params, U=U0)
    n = run.run(10.0)
    ref_steps = len(ref.steps(100000, 10.0)[0])
    assert n == ref_steps == 1498
    U = run.state()
    assert bits_equal(U, ref.state())
    assert run.t == ref.t
    # one period later the exact solution is the initial state
    err = math.sqrt(np.mean((U[:, 0] - U0[:, 0]) ** 2))
    assert err < 2e-3, err


def test_c3_riemann_quadrants_reduced():
    n = 192
    params = dict(nx=n, ny=n, Lx=1.0, Ly=1.0, reconstruction="weno5", riemann_solver="HLLC", time_scheme="SSP Runge-Kutta 3", cfl=0.4,
                  **cases.bcs("transmissive", "transmissive", "transmissive", "transmissive"))
    U0 = quadrants(n, 2024)
    ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
    ref.set_state(U0)
    run = Run(params, U=U0)
    steps = run.run(0.25)
    assert steps == len(ref.steps(100000, 0.25)[0])
    assert bits_equal(run.state(), ref.state())
    assert run.t == ref.t == 0.25


def test_c2_taylor_green_reduced():
    n = 48
    L = 2 * math.pi
    params = dict(nx=n, ny=n, nz=n, Lx=L, Ly=L, Lz=L, use_viscous=True, mu=6.25e-4, pr=0.71, reconstruction="weno5",
                  riemann_solver="HLLC (Low-Mach Thornber)", time_scheme="SSP Runge-Kutta 3", cfl=0.5,
                  **cases.bcs("periodic", "periodic", "periodic", "periodic"))
    ref = Reference(params, initial_profile="taylor_green_3d")
    run = Run(params, U=ref.state())
    assert run.run(1e30, max_steps=10) == 10
    ref.steps(10, 1e30)
    assert bits_equal(run.state(), ref.state())
    assert run.t == ref.t
