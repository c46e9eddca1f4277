"""The slab decomposition on one GPU: the mesh split into 2 to 4 parts held by one process (LocalExchange: the parts'
interface planes and all-reduced wave speeds copied between them in the order fvg_part_phase asks), run for a few steps,
equals the whole run bit for bit (state, t, step count), for 2-D and 3-D meshes, every time scheme, the viscous sweep,
the body force, periodic and wall sides on the split axis, uneven splits, and the mixed-precision form; and the part
configurations the library refuses."""
import numpy as np
import pytest

import cases
from fenice_b200 import Run, initial, slabs

pytestmark = pytest.mark.gpu

B = cases.bcs
TGV = dict(Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, **B("periodic", "periodic", "periodic", "periodic"))
SLAB_CASES = [
    ("w5_rk3_visc_periodic_3d", dict(nx=20, ny=18, nz=16, reconstruction="weno5", riemann_solver="lowmach", time_scheme="SSP Runge-Kutta 3",
                                     use_viscous=True, mu=0.01, **TGV), 61, 4, (2, 3), 0),
    ("muscl_rk2_walls_z_3d", dict(nx=12, ny=10, nz=13, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2",
                                  **B("transmissive", "outlet", "periodic", "periodic", z=("wall", "no_slip"))), 62, 4, (3,), 0),
    ("hancock_visc_periodic_3d", dict(nx=16, ny=12, nz=12, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="MUSCL-Hancock",
                                      use_viscous=True, mu=0.02, **TGV), 63, 5, (2, 4), 0),
    ("w3_rk3_order1_walls_3d", dict(nx=10, ny=9, nz=11, reconstruction="weno3", boundary_order=1, time_scheme="SSP Runge-Kutta 3",
                                    use_viscous=True, mu=0.01, **B("no_slip", "transmissive", "wall", "moving_wall", z=("moving_wall", "wall")),
                                    u_in=0.3, v_in=0.1), 64, 3, (2,), 0),
    ("w5_rk3_inlet_2d", dict(nx=40, ny=33, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", **B("vel_inlet", "transmissive", "wall", "outlet"),
                             u_in=0.8, p_out=0.9), 65, 4, (3,), 0),
    ("hancock_grav_2d", dict(nx=30, ny=24, reconstruction="muscl", muscl_limiter="Koren", time_scheme="MUSCL-Hancock", use_bodyforce=True,
                             gy=-1.5, **B("periodic", "periodic", "wall", "wall")), 66, 5, (2, 4), 0),
    ("visc_rk3_walls_2d", dict(nx=28, ny=26, reconstruction="muscl", muscl_limiter="Minmod", time_scheme="SSP Runge-Kutta 3", use_viscous=True,
                               mu=0.02, **B("no_slip", "no_slip", "no_slip", "moving_wall"), u_in=0.5), 67, 4, (2,), 0),
    ("first_order_euler_2d", dict(nx=25, ny=20, reconstruction="none", time_scheme="Explicit Euler", **B("wall", "outlet", "transmissive", "wall")),
     68, 5, (3,), 0),
    ("w5_rk3_periodic_2d", dict(nx=32, ny=30, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", **B("periodic", "periodic", "periodic", "periodic")),
     69, 4, (1, 2, 3), 0),
    ("mixed_w5_rk3_visc_3d", dict(nx=20, ny=16, nz=18, reconstruction="weno5", riemann_solver="lowmach", time_scheme="SSP Runge-Kutta 3",
                                  use_viscous=True, mu=0.01, **TGV), 70, 4, (2, 3), 1),
    # the whole run's mixed WENO5-Z kernel stages its interior tiles by TMA; the parts' kernels load every tile by index mapping
    ("mixed_w5_rk3_visc_64_tma", dict(nx=64, ny=64, nz=64, reconstruction="weno5", riemann_solver="lowmach", time_scheme="SSP Runge-Kutta 3",
                                      use_viscous=True, mu=0.01, **TGV), 72, 4, (1, 2), 1),
    # non-reflecting outlets: on x, whose tangential z neighbours cross the part interfaces, and at the low z end
    ("nrbc_w5_rk3_visc_3d", dict(nx=12, ny=10, nz=13, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", use_viscous=True, mu=0.01,
                                 **B("transmissive", "nonreflecting", "periodic", "periodic", z=("nonreflecting", "wall"))), 71, 3, (2, 3), 0),
]


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


@pytest.mark.parametrize("case", SLAB_CASES, ids=[c[0] for c in SLAB_CASES])
def test_decomposed_run_equals_whole_run(case):
    name, params, seed, n, nparts_list, precision = case
    U0 = cases.case_field(params, seed)
    whole = Run(params, U=U0, precision=precision)
    assert whole.run(1e30, max_steps=n) == n
    Uw, tw = whole.state(), whole.t
    whole.close()
    for nparts in nparts_list:
        U, steps, t = slabs.run_decomposed(params, U0, nparts, 1e30, max_steps=n, precision=precision)
        assert steps == n
        assert t == tw, (nparts, t, tw)
        d = np.abs(U - Uw)
        assert bits_equal(U, Uw), f"{nparts} parts: max |diff| {d.max():.3e}, {int((d > 0).sum())} values differ"


def test_decomposed_run_to_t_end():
    """A run to t_end (the last step clamped) ends at the same time and state in 3 parts."""
    params = dict(SLAB_CASES[0][1])
    U0 = initial.taylor_green_3d(20)[: 20 * 20 * 20]
    params.update(nx=20, ny=20, nz=20)
    whole = Run(params, U=U0)
    steps_w = whole.run(0.05)
    Uw, tw = whole.state(), whole.t
    U, steps, t = slabs.run_decomposed(params, U0, 3, 0.05)
    assert steps == steps_w and t == tw == 0.05
    assert bits_equal(U, Uw)


@pytest.mark.parametrize("params,nparts,words", [
    (dict(nx=16, ny=16, nz=4, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", **TGV), 2, "at least 3 planes"),
    (dict(nx=16, ny=12, reconstruction="none", time_scheme="Explicit Euler", **B("periodic", "periodic", "periodic", "periodic")), 2, "periodic axis"),
    (dict(nx=32, ny=24, Lx=4.0, Ly=3.0, use_ibm=True, ibm_radius=0.3, ibm_cx=1.0, ibm_cy=1.5, reconstruction="muscl", u_in=0.5,
          **B("vel_inlet", "transmissive", "wall", "wall")), 2, "immersed body"),
    (dict(nx=32, ny=24, reconstruction="muscl", time_scheme="SSP Runge-Kutta 2", u_in=0.5, **B("massflow_inlet", "outlet", "wall", "wall")), 2,
     "mass-flow inlet"),
])
def test_part_refusals(params, nparts, words):
    with pytest.raises(ValueError, match=words):
        slabs.Part(params, nparts, 0)


def test_part_refuses_whole_run_entry_points():
    params = dict(SLAB_CASES[0][1])
    p = slabs.Part(params, 2, 0, U=slabs.split_state(params, cases.case_field(params, 61), 2)[0])
    with pytest.raises(ValueError, match="fvg_part_phase"):
        p.run(1e30, max_steps=1)
    with pytest.raises(ValueError, match="fvg_part_phase"):
        p.residual()
    p.close()


def test_gated_mixed_form_decomposed():
    """The mixed form gated by the learned sensor on a decomposed mesh (2 parts of a periodic 64^3 Taylor-Green box, the
    refresh every 5 steps after each part's interface planes arrive): the tile rows whose gate box reaches an interface
    stay WENO5-Z along every axis, the other tiles take the flags the whole run takes from the same state, and the
    totals stay conserved (the interface faces are solved alike by both parts)."""
    import math
    import os

    import bench
    from fenice_b200.sensor import Sensor

    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    s = Sensor.load(os.path.join(here, "fenice_b200", "sensor_weights.npz"), device=0)
    theta = float(s.meta["threshold"])
    n, nparts, every = 64, 2, 5
    params = bench.workload(n)
    U0 = bench.tgv_state(n)
    whole = Run(params, U=U0, precision=1)
    whole.set_sensor(s, theta, every=every)
    assert whole.run(1e30, max_steps=1) == 1
    _, wt, tile = whole.sensor_gate()
    parts = [slabs.Part(params, nparts, i, U=u, precision=1) for i, u in enumerate(slabs.split_state(params, U0, nparts))]
    try:
        for p in parts:
            p.set_sensor(s, theta, every=every)
        ex = slabs.LocalExchange(parts)
        slabs.advance(parts, ex, 1e30, 1)
        radius = int(math.ceil(0.5 * every)) + 1
        tz = tile[2]
        for p in parts:
            _, pt, _ = p.sensor_gate()
            rows = pt.shape[1]
            for r in range(rows):
                lo, hi = r * tz, min((r + 1) * tz, p.count) - 1
                reaches = lo - (radius + 1) < 0 or hi + radius + 1 > p.count - 1
                if reaches:
                    assert np.all(pt[:, r] == 1), (p.index, r)
                else:
                    assert np.array_equal(pt[:, r], wt[:, (p.first + lo) // tz]), (p.index, r)
        steps, _ = slabs.advance(parts, ex, 1e30, 20)   # (the step count and the refresh cadence start again per call)
        assert steps == 20
        U = slabs.join_states(params, [p.state() for p in parts])
        lin, ev = parts[0].sensor_counts()
        assert 0 < lin < ev
    finally:
        for p in parts:
            p.close()
        whole.close()
    mom = math.fsum(np.sqrt(U0[:, 1] ** 2 + U0[:, 2] ** 2 + U0[:, 4] ** 2))
    scale = np.array([math.fsum(np.abs(U0[:, 0])), mom, mom, math.fsum(np.abs(U0[:, 3])), mom])
    drift = np.array([abs(math.fsum(U[:, q]) - math.fsum(U0[:, q])) for q in range(5)]) / scale
    print(f"\ngated, 2 parts, 21 steps: {lin} of {ev} tile-axes linear on part 0; drift of the totals " + " ".join(f"{d:.1e}" for d in drift))
    assert np.all(drift <= 2e-11)
