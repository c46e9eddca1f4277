"""fvg_step_host: one step of a state held in host memory (the reference's TimeScheme::step(Field& U, ...) seam, whose
caller owns U). The pipelined form uploads the state in slabs along the slowest axis while the first stage runs on the
slabs that have arrived, and reads the last stage back slab by slab; it must give the bits of upload + fvg_step +
download (which the parity tests pin to the reference) on every kind of run: 3-D and 2-D, periodic and bounded axes,
slabs that do not line up with the stage tiles, viscous and inviscid, Euler / SSP-RK2 / SSP-RK3, FP64 and mixed
precision, the learned sensor's gate, and the runs that take the unpipelined route (an immersed body)."""
import math

import numpy as np
import pytest

import cases
from fenice_b200 import Run
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

L2PI = 2 * math.pi
TGV = dict(Lx=L2PI, Ly=L2PI, Lz=L2PI, use_viscous=True, mu=6.25e-4, pr=0.71, reconstruction="weno5", riemann_solver="lowmach",
           time_scheme="SSP Runge-Kutta 3", cfl=0.5, **cases.bcs("periodic", "periodic", "periodic", "periodic"))


def tgv(nx, ny, nz):
    h = (L2PI / nx, L2PI / ny, L2PI / nz)
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) * h[2], (np.arange(ny) + 0.5) * h[1], (np.arange(nx) + 0.5) * h[0], indexing="ij")
    u = (np.sin(x) * np.cos(y) * np.cos(z)).ravel()
    v = (-np.cos(x) * np.sin(y) * np.cos(z)).ravel()
    p = (1.0 / (1.4 * 0.01) + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0).ravel()
    W = np.stack([np.ones_like(u), u, v, p, np.zeros_like(u)], axis=1)
    return cases.prim_to_cons(W)


CYLP = dict(nx=64, ny=96, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4, **cases.CYL)
CASES = [
    # 64 z planes: 8 slabs of one tile plane each, the first uploaded last-slab-first (periodic z)
    ("tgv3d_fp64_rk3_viscous", dict(nx=24, ny=16, nz=64, **TGV), lambda: tgv(24, 16, 64), 3, 0),
    ("tgv3d_mixed_rk3_viscous", dict(nx=24, ny=16, nz=64, **TGV), lambda: tgv(24, 16, 64), 3, 1),
    # 2-D, bounded y: 200 rows in 16 slabs of 13, stage tiles 15 rows high (tile planes straddle slabs)
    ("riemann2d_fp64_weno5_rk3", dict(nx=40, ny=200, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4,
                                      **cases.bcs("transmissive", "transmissive", "transmissive", "transmissive")),
     lambda: cases.smooth_field(40, 200, seed=11, jump=True), 3, 0),
    ("walls2d_visc_muscl_rk2", dict(nx=48, ny=96, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2", use_viscous=True,
                                    mu=2e-3, **cases.bcs("wall", "outlet", "no_slip", "vel_inlet"), u_in=0.2),
     lambda: cases.smooth_field(48, 96, seed=5), 3, 0),
    ("box3d_weno3_euler_walls", dict(nx=16, ny=16, nz=40, Lz=2.5, reconstruction="weno3", time_scheme="Euler", cfl=0.3,
                                     **cases.bcs("wall", "wall", "transmissive", "transmissive", z=("wall", "transmissive"))),
     lambda: cases.smooth_field(16, 16, 40, seed=2), 2, 0),
    # a run the overlap does not cover: the three calls in turn
    ("cylinder_ibm_rk3", CYLP, lambda: cases.ibm_field(CYLP, (1.4, 2.0, 0.0, 1.0), 42), 2, 0),
]


def reference_steps(params, U0, n, precision):
    """upload + fvg_step + download, n times"""
    run = Run(params, U=U0, precision=precision, device=0)
    U = U0.copy()
    dts = []
    for _ in range(n):
        run.set_state(U)
        dts.append(run.step(1e30))
        U = run.state()
    run.close()
    return U, dts


@pytest.mark.parametrize("name,params,init,n,precision", CASES, ids=[c[0] for c in CASES])
def test_step_host_equals_upload_step_download(name, params, init, n, precision):
    U0 = init()
    want, want_dt = reference_steps(params, U0, n, precision)
    run = Run(params, U=U0, precision=precision, device=0)
    U = U0.copy()
    got_dt = [run.step_host(U, 1e30) for _ in range(n)]   # in place
    assert got_dt == want_dt
    assert np.array_equal(U.view(np.uint64), want.view(np.uint64)), f"{name}: max |diff| {np.abs(U - want).max():.3e}"
    # into a separate array, from pinned memory
    torch = pytest.importorskip("torch")
    src = torch.empty(U0.shape, dtype=torch.float64, pin_memory=True).numpy()
    dst = torch.empty(U0.shape, dtype=torch.float64, pin_memory=True).numpy()
    src[:] = want
    run2 = Run(params, U=want, precision=precision, device=0)
    run2.set_state(want)
    r1 = run2.step(1e30)
    after = run2.state()
    r2 = run.step_host(src, 1e30, out=dst)
    assert r1 == r2
    assert np.array_equal(dst.view(np.uint64), after.view(np.uint64))
    assert np.array_equal(src.view(np.uint64), want.view(np.uint64))   # the input is left alone
    run.close()
    run2.close()


def test_step_host_against_the_oracle():
    params = dict(nx=32, ny=80, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4,
                  **cases.bcs("periodic", "periodic", "transmissive", "wall"))
    U0 = cases.case_field(params, 9)
    run = Run(params, U=U0, device=0)
    U = U0.copy()
    for _ in range(2):
        run.step_host(U, 1e30)
    want, t, _, _, _ = Oracle().run(params, U0, 2)
    assert np.array_equal(U.view(np.uint64), want.view(np.uint64))
    assert run.t == t
    run.close()


def test_step_host_with_the_sensor_matches_the_graph_run():
    """The gate refreshed every `every` calls, as the graph-launched run refreshes it every `every` steps."""
    pytest.importorskip("torch")
    from fenice_b200.sensor import Sensor

    params = dict(nx=24, ny=16, nz=64, **TGV)
    U0 = tgv(24, 16, 64)
    s = Sensor(seed=3)
    graph = Run(params, U=U0, precision=1, device=0)
    graph.set_sensor(s, 0.0, every=3)
    assert graph.run(1e30, max_steps=7) == 7
    want = graph.state()
    lin_g, ev_g = graph.sensor_counts()
    host = Run(params, U=U0, precision=1, device=0)
    host.set_sensor(s, 0.0, every=3)
    U = U0.copy()
    for _ in range(7):
        host.step_host(U, 1e30)
    assert np.array_equal(U.view(np.uint64), want.view(np.uint64))
    assert host.sensor_counts() == (lin_g, ev_g)
    graph.close()
    host.close()


def test_step_host_past_the_end_leaves_the_state():
    params = dict(nx=24, ny=16, nz=64, **TGV)
    U0 = tgv(24, 16, 64)
    run = Run(params, U=U0, device=0)
    U = U0.copy()
    r = run.step_host(U, 0.0)
    assert r.dt == 0.0
    assert np.array_equal(U.view(np.uint64), U0.view(np.uint64))
    run.close()


def test_step_host_refuses_rho_w_on_a_2d_mesh():
    params = dict(nx=32, ny=32, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", **cases.bcs("periodic", "periodic", "periodic", "periodic"))
    U0 = cases.case_field(params, 1)
    run = Run(params, U=U0, device=0)
    bad = U0.copy()
    bad[5, 4] = 0.1
    with pytest.raises(ValueError, match="rho w"):
        run.step_host(bad, 1e30)
    with pytest.raises(ValueError, match="shape"):
        run.step_host(U0[:-1], 1e30)
    run.close()
