"""Conservation of mass, momentum and energy on periodic meshes, in every form: the plain FP64 form, the mixed form
(FP32 stencil, flux and balance; FP64 state) and the mixed form gated by the learned sensor (with its refreshes).

On a periodic mesh every face flux leaves one cell and enters another, so the totals of rho, rho u, rho v, rho w and
rho E change only by rounding (the reference's balance, cpp/src/Schemes.cpp:1125-1170, telescopes the same way). That
requires each face to be solved identically by the two tiles that share it: in the gated form a seam face between a
linear and a WENO5-Z tile takes WENO5-Z from both.

Bounds, relative to the sum over the cells of |rho|, of |rho E| and, for every momentum component, of the momentum's
magnitude (a component whose total starts at 0, such as the Taylor-Green rho w, is measured against the momentum scale):
- plain FP64: 1e-13 (each stage rounds per cell at about 1e-16 of |U|; the sum of N such errors is ~ sqrt(N) of one;
  measured 3e-15 after 50 steps);
- mixed and gated: the per-cell flux differences and their balance are rounded in FP32 (6e-8 of each difference) before
  the FP64 update. In smooth flow the differences are O(h) of the fluxes: bound 2e-11 on the Taylor-Green boxes (measured
  up to 4e-12 after 50 steps). Across a jump a difference is O(1) of the flux: bound 5e-10 on the jump boxes (measured up
  to 1.5e-10, mixed and gated alike).
A seam face solved differently by the two tiles that share it (a linear reconstruction on one side, WENO5-Z on the other)
moves the totals by the difference of the two reconstructions at every stage: measured with such a kernel, 1e-10 to
1e-9 on the Taylor-Green boxes and 1.4e-9 to 4.1e-9 on the jump boxes, beyond both bounds. The totals are taken with
math.fsum (exactly rounded), so the check sees the solver's drift only.
"""
import math
import os

import numpy as np
import pytest

import cases
from fenice_b200 import Run

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 50
# (form, smooth flow) -> bound on the relative drift of every total
BOUND = {("plain", True): 1e-13, ("plain", False): 1e-13, ("mixed", True): 2e-11, ("mixed", False): 5e-10, ("gated", True): 2e-11,
         ("gated", False): 5e-10}


def totals(U):
    return np.array([math.fsum(U[:, q]) for q in range(U.shape[1])])


def tgv_case(n):
    import bench

    params = dict(nx=n, ny=n, nz=n, Lx=2 * math.pi, Ly=2 * math.pi, Lz=2 * math.pi, use_viscous=True, mu=6.25e-4, pr=0.71,
                  reconstruction="weno5", riemann_solver="lowmach", time_scheme="SSP Runge-Kutta 3", cfl=0.5,
                  **cases.bcs("periodic", "periodic", "periodic", "periodic"))
    return params, bench.tgv_state(n)


def jump_box(nx, ny, seed):
    """Four seeded constant quadrants on a periodic box: jumps along x = 1/2, y = 1/2 and across the periodic sides."""
    rng = np.random.default_rng(seed)
    st = [(rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.1, 2)) for _ in range(4)]
    y, x = np.meshgrid((np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx, indexing="ij")
    x, y = x.ravel(), y.ravel()
    q = np.where(x >= 0.5, np.where(y >= 0.5, 0, 3), np.where(y >= 0.5, 1, 2))
    W = np.zeros((nx * ny, 5))
    for k, (r, u, v, p) in enumerate(st):
        W[q == k] = (r, u, v, p, 0.0)
    params = dict(nx=nx, ny=ny, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4,
                  **cases.bcs("periodic", "periodic", "periodic", "periodic"))
    return params, cases.prim_to_cons(W)


CASES = [
    ("tgv3d_64", lambda: tgv_case(64)),
    ("tgv3d_60", lambda: tgv_case(60)),          # partial tiles at the periodic ends
    ("jumpbox2d_128", lambda: jump_box(128, 128, 11)),
    ("jumpbox2d_200x136", lambda: jump_box(200, 136, 12)),
]


def sensor():
    from fenice_b200.sensor import Sensor

    return Sensor.load(os.path.join(HERE, "fenice_b200", "sensor_weights.npz"), device=0)


@pytest.mark.parametrize("form", ["plain", "mixed", "gated"])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_totals_conserved(name, make, form):
    params, U0 = make()
    run = Run(params, U=U0, precision=0 if form == "plain" else 1)
    if form == "gated":
        s = sensor()
        run.set_sensor(s, float(s.meta["threshold"]), every=5)
    assert run.run(1e30, max_steps=STEPS) == STEPS
    U = run.state()
    nv = 5 if params.get("nz", 1) > 1 else 4
    mom = math.fsum(np.sqrt(U0[:, 1] ** 2 + U0[:, 2] ** 2 + U0[:, 4] ** 2))
    scale = np.array([math.fsum(np.abs(U0[:, 0])), mom, mom, math.fsum(np.abs(U0[:, 3])), mom][:nv])
    drift = np.abs(totals(U[:, :nv]) - totals(U0[:, :nv])) / scale
    msg = f"\n{name} {form}: relative drift of the totals after {STEPS} steps " + " ".join(f"{d:.1e}" for d in drift)
    if form == "gated":
        lin, ev = run.sensor_counts()
        msg += f"; gate {lin} of {ev} tile-axes linear"
        # the jump boxes put linear and WENO5-Z tiles side by side (the seams the check is about); the Taylor-Green
        # boxes are smooth and pass linear
        assert (0 < lin < ev) if name.startswith("jump") else lin > 0
    print(msg)
    assert np.all(drift <= BOUND[(form, name.startswith("tgv"))]), drift
    run.close()
