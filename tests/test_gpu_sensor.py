"""The learned troubled-cell sensor on the GPU against its CPU oracle (oracle/sensor_oracle.py): the tensor-core
forward pass (logits), the backward pass (every gradient), the training data (features and label statistics of a run's
state), and that Adam on the GPU kernels learns the label."""
import numpy as np
import pytest

from fenice_b200 import Run, initial
from fenice_b200.sensor import TAU
from oracle import sensor_oracle as SO

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def sensor(seed=0):
    from fenice_b200.sensor import Sensor

    return Sensor(seed=seed)


def random_params(seed):
    rng = np.random.default_rng(seed)
    P = {"W1": rng.normal(0, 0.4, (32, 32)), "b1": rng.normal(0, 0.2, 32), "W2": rng.normal(0, 0.3, (32, 32)), "b2": rng.normal(0, 0.2, 32),
         "w3": rng.normal(0, 0.3, 32), "b3": 0.1}
    P["W1"][:, 25:] = 0.0
    return P


def random_features(n, seed):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, 32), dtype=np.float32)
    X[:, :25] = rng.uniform(-1, 1, (n, 25))
    X[:, 2:25:5] = rng.uniform(0, 4, (n, 5))
    return X


def test_forward_matches_oracle():
    from fenice_b200.sensor import Sensor

    P = random_params(1)
    s = Sensor(params=P)
    X = random_features(4099, 2)
    z = s.logits(torch.tensor(X, device="cuda")).cpu().numpy()
    zr, _ = SO.mlp_forward(X, P)
    close = np.isclose(z, zr, rtol=1e-3, atol=2e-3)
    print(f"\nforward: max |dz| {np.abs(z - zr).max():.2e}, {close.mean():.4f} within tolerance")
    assert close.mean() > 0.995


def test_gradients_match_oracle():
    from fenice_b200.sensor import Sensor

    P = random_params(3)
    s = Sensor(params=P)
    n = 3001
    X = random_features(n, 4)
    y = (np.random.default_rng(5).random(n) < 0.3).astype(np.float32)
    loss, g = s.grad(torch.tensor(X, device="cuda"), torch.tensor(y, device="cuda"), wpos=3.0)
    G = Sensor.unflatten(g.cpu().numpy().astype(np.float64))
    lr, Gr = SO.mlp_loss_grad(X, y, 3.0, P)
    assert abs(loss - lr) <= 1e-3 * abs(lr)
    for k in ("W1", "b1", "W2", "b2", "w3", "b3"):
        a, b = np.asarray(G[k]), np.asarray(Gr[k])
        if k == "W1":
            a, b = a[:, :25], b[:, :25]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        print(f"grad {k}: relative error {rel:.2e}")
        assert rel < 1e-2, k


def stencils(W, n, axis):
    """(n*n, 5, 5) stencils along `axis` of interior-padded primitive cells (only interior cells are compared)."""
    Wg = W.reshape(n, n, 5)
    out = np.zeros((n, n, 5, 5))
    for k in range(-2, 3):
        out[:, :, k + 2] = np.roll(Wg, -k, axis=1 - axis)
    return out.reshape(n * n, 5, 5)


def test_training_data_matches_oracle():
    from fenice_b200.sensor import Sensor

    n = 48
    run = Run(initial.quadrant_params(n), U=initial.riemann_quadrants(n, 9))
    run.run(0.05)
    U = run.state()
    s = Sensor()
    X, D, stats = s.samples(run, mode=0)
    X, D = X.cpu().numpy().reshape(n * n, 2, 32), D.cpu().numpy().reshape(n * n, 2)
    g = 1.4
    W = np.zeros((n * n, 5))
    W[:, 0] = U[:, 0]
    W[:, 1], W[:, 2] = U[:, 1] / U[:, 0], U[:, 2] / U[:, 0]
    W[:, 3] = (g - 1) * (U[:, 3] - 0.5 * (U[:, 1] ** 2 + U[:, 2] ** 2) / U[:, 0])
    inner = np.zeros((n, n), bool)
    inner[2:-2, 2:-2] = True
    inner = inner.ravel()
    for axis in (0, 1):
        Q = SO.axis_quantities(stencils(W, n, axis), axis)
        Xr, Dr = SO.stencil_features(Q), SO.departure(Q)
        assert np.allclose(X[inner, axis], Xr[inner], rtol=1e-4, atol=1e-4), np.abs(X[inner, axis] - Xr[inner]).max()
        # the statistic is a difference of two face values (rounding of values of order 1 against scales of order 0.1)
        assert np.allclose(D[inner, axis], Dr[inner], rtol=1e-4, atol=1e-12), np.abs(D[inner, axis] - Dr[inner]).max()
    assert stats[1] == n * n * 2 and stats[0] == int((D > TAU).sum())


def test_adam_on_the_gpu_learns_the_label():
    from fenice_b200.sensor import Sensor, quadrant_training_data

    s = Sensor(seed=7)
    X, D = quadrant_training_data(s, seeds=[1, 2, 3], n=128, t_end=0.2, snapshots=3)
    y = (D > TAU).float()
    before = s.grad(X, y, wpos=1.0)[0]
    losses = s.train(X, y, epochs=6, batch=4096, lr=3e-3)
    after = s.grad(X, y, wpos=1.0)[0]
    acc = ((s.logits(X) > 0).float() == y).float().mean().item()
    print(f"\n{len(X)} samples, troubled {y.mean().item():.3f}; loss {before:.4f} -> {after:.4f} (epochs {[round(v, 4) for v in losses]}); "
          f"accuracy {acc:.4f}")
    assert after < 0.5 * before and acc > 0.9


def test_gate_extremes_and_counts():
    """With a threshold no logit reaches from below every reconstruction stays WENO5-Z: the gated run gives the plain
    mixed run's state (to FP32 rounding: the gated kernel is compiled separately); with one every logit is below, every
    tile away from the transmissive sides takes the linear reconstruction and the run differs."""
    from fenice_b200.sensor import Sensor

    n = 96
    params, U0 = initial.quadrant_params(n), initial.riemann_quadrants(n, 4)
    plain = Run(params, U=U0, precision=1)
    plain.run(0.05)
    s = Sensor(seed=3)
    weno = Run(params, U=U0, precision=1)
    weno.set_sensor(s, -1e30, every=3)
    weno.run(0.05)
    d = np.abs(weno.state() - plain.state()).max()
    lin, ev = weno.sensor_counts()
    print(f"\ngate all WENO5-Z: max |diff| vs plain {d:.2e}, counts {lin}/{ev}")
    assert d <= 1e-5 and lin == 0 and ev > 0
    linear = Run(params, U=U0, precision=1)
    linear.set_sensor(s, 1e30, every=3, radius=0)
    linear.run(0.05)
    lin, ev = linear.sensor_counts()
    tiles_x, tiles_y = -(-n // 16), -(-n // 15)
    inner = (tiles_x - 2) * tiles_y + tiles_x * (tiles_y - 2)   # x sweeps: tiles off the x sides; y sweeps: off the y sides
    print(f"gate all linear: counts {lin}/{ev} per refresh pattern, interior tile-axes {inner}")
    assert lin > 0 and lin % inner == 0 and np.abs(linear.state() - plain.state()).max() > 0


GATE_CASES = [
    # (name, mesh and boundaries, initial state, refresh period, dilation radius (-1: ceil(cfl every) + 1))
    ("tgv3d_48_periodic", dict(nx=48, ny=48, nz=48, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, use_viscous=True, mu=6.25e-4, pr=0.71,
                               reconstruction="weno5", riemann_solver="lowmach", time_scheme="SSP Runge-Kutta 3", cfl=0.5,
                               bc_xmin="periodic", bc_xmax="periodic", bc_ymin="periodic", bc_ymax="periodic", bc_zmin="periodic",
                               bc_zmax="periodic"), "tgv", 5, -1),
    ("box3d_mixed_sides_r3", dict(nx=40, ny=36, nz=28, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4, bc_xmin="periodic",
                                  bc_xmax="periodic", bc_ymin="transmissive", bc_ymax="wall", bc_zmin="periodic", bc_zmax="periodic"), "jump", 4, 3),
    ("quadrants2d_200x136_r6", dict(nx=200, ny=136, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4, bc_xmin="transmissive",
                                    bc_xmax="transmissive", bc_ymin="transmissive", bc_ymax="transmissive"), "quadrants", 5, 6),
    ("periodic2d_96x80_r2", dict(nx=96, ny=80, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4, bc_xmin="periodic",
                                 bc_xmax="periodic", bc_ymin="periodic", bc_ymax="periodic"), "jump", 3, 2),
]


@pytest.mark.parametrize("name,params,init,every,radius", GATE_CASES, ids=[c[0] for c in GATE_CASES])
def test_gate_matches_the_oracle(name, params, init, every, radius):
    """The tile flags the stage kernels read, from the network's flags of the same refresh through the oracle's
    dilation and tile reduction: identical."""
    import os
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    import cases
    from fenice_b200.sensor import Sensor

    if init == "tgv":
        import bench

        U0 = bench.tgv_state(params["nx"])
    elif init == "quadrants":
        U0 = initial.riemann_quadrants(params["nx"], 4) if params["nx"] == params["ny"] else cases.case_field(params, 6)
    else:
        U0 = cases.case_field(params, 6)
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    s = Sensor.load(os.path.join(here, "fenice_b200", "sensor_weights.npz"), device=0)
    run = Run(params, U=U0, precision=1)
    run.set_sensor(s, float(s.meta["threshold"]), every=every, radius=radius)
    assert run.run(1e30, max_steps=1) == 1
    cells, tiles, tile = run.sensor_gate()
    dim = cells.shape[0]
    nz = int(params.get("nz", 1))
    per = [params.get(f"bc_{a}min") == "periodic" and params.get(f"bc_{a}max") == "periodic" for a in "xyz"]
    r = radius if radius >= 0 else int(np.ceil(params["cfl"] * every)) + 1
    want = SO.gate_tiles(cells.reshape(dim, nz, params["ny"], params["nx"]), tile, r, per)
    lin = int((tiles == 0).sum())
    print(f"\n{name}: {int(cells.sum())} of {cells.size} (cell, axis) pairs flagged, {lin} of {tiles.size} tile-axes linear")
    assert np.array_equal(tiles, want)
    run.close()
