"""The slab decomposition across processes: two processes, each driving one part of the mesh on the same GPU and
exchanging their interface planes and all-reduced speeds through pinned host memory over a gloo process group
(fenice_b200.slabs.HostStagedExchange: every wait is on the host, no kernel waits for the other process). The joined
state equals the whole run bit for bit (plain FP64 and mixed forms), and, for the mixed form gated by the learned
sensor, the same decomposition run in one process (LocalExchange)."""
import datetime
import os
import socket
import tempfile

import numpy as np
import pytest

import cases
from fenice_b200 import Run, slabs

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def sensor():
    from fenice_b200.sensor import Sensor

    s = Sensor.load(os.path.join(HERE, "fenice_b200", "sensor_weights.npz"), device=0)
    return s, float(s.meta["threshold"])


def _rank(rank, world, port, params, states, steps, precision, gated, out):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        part = slabs.Part(params, world, rank, U=states[rank], precision=precision, device=0)
        if gated:
            part.set_sensor(*sensor())
        done, t = slabs.advance([part], slabs.HostStagedExchange(part), 1e30, steps, check_every=4)
        np.savez(os.path.join(out, f"rank{rank}.npz"), U=part.state(), t=t, steps=done)
        part.close()
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def two_processes(params, U0, steps, precision, gated):
    import torch.multiprocessing as mp

    world = 2
    out = tempfile.mkdtemp(prefix="fvg_mp_")
    mp.start_processes(_rank, args=(world, free_port(), params, slabs.split_state(params, U0, world), steps, precision, gated, out), nprocs=world,
                       join=True, start_method="spawn")
    res = [np.load(os.path.join(out, f"rank{r}.npz")) for r in range(world)]
    assert all(float(r["t"]) == float(res[0]["t"]) and int(r["steps"]) == int(res[0]["steps"]) for r in res)
    return slabs.join_states(params, [r["U"] for r in res]), float(res[0]["t"]), int(res[0]["steps"])


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


CASES = [
    ("w5_rk3_visc_periodic_3d", dict(nx=20, ny=18, nz=16, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, reconstruction="weno5", riemann_solver="lowmach",
                                     time_scheme="SSP Runge-Kutta 3", use_viscous=True, mu=0.01, **cases.bcs("periodic", "periodic", "periodic", "periodic")),
     61, 6, 0),
    ("w5_rk3_inlet_2d", dict(nx=40, ny=33, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", **cases.bcs("vel_inlet", "transmissive", "wall", "outlet"),
                             u_in=0.8, p_out=0.9), 65, 6, 0),
    ("mixed_w5_rk3_visc_walls_3d", dict(nx=16, ny=16, nz=20, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", use_viscous=True, mu=0.01,
                                        **cases.bcs("transmissive", "transmissive", "periodic", "periodic", z=("wall", "no_slip"))), 70, 6, 1),
]


@pytest.mark.timeout(600)
@pytest.mark.parametrize("name,params,seed,steps,precision", CASES, ids=[c[0] for c in CASES])
def test_two_processes_equal_the_whole_run(name, params, seed, steps, precision):
    U0 = cases.case_field(params, seed)
    U, t, done = two_processes(params, U0, steps, precision, False)
    whole = Run(params, U=U0, precision=precision)
    assert whole.run(1e30, max_steps=steps) == steps == done
    assert bits_equal(U, whole.state()) and t == whole.t
    whole.close()


@pytest.mark.timeout(600)
def test_two_processes_gated_equal_the_same_decomposition_in_one_process():
    import bench

    n, steps = 48, 12
    params, U0 = bench.workload(n), bench.tgv_state(n)
    U, t, done = two_processes(params, U0, steps, 1, True)
    parts = [slabs.Part(params, 2, i, U=u, precision=1) for i, u in enumerate(slabs.split_state(params, U0, 2))]
    s = sensor()
    for p in parts:
        p.set_sensor(*s)
    got, t1 = slabs.advance(parts, slabs.LocalExchange(parts), 1e30, steps)
    Ul = slabs.join_states(params, [p.state() for p in parts])
    for p in parts:
        p.close()
    assert got == done == steps and t1 == t
    assert bits_equal(U, Ul)
