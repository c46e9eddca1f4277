"""Trains the learned troubled-cell sensor on the GPU and writes its weights (fenice_b200/sensor_weights.npz).

    python -m fenice_b200.train_sensor [--out PATH] [--seeds 64] [--n 512]

Training data (labels from plain WENO5-Z runs in FP64, the reference's arithmetic): 64 seeded four-quadrant Riemann
problems at 512^2 (WENO5-Z + HLLC + SSP-RK3, CFL 0.4, to t = 0.25, 4 snapshots), 8 seeded eight-octant problems at 64^3
(every troubled (cell, axis) pair, a WENO5-Z face value more than 1e-5 of the quantity's scale from the linear one, and
every 16th other one) and the 3-D Taylor-Green vortex at 64^3 (Re 1600, steps 3, 10, 40, 100 and 200) and 128^3 (steps
3 and 20), every 4th pair. Adam on the library's
tensor-core forward and backward kernels. Held-out data (4 quadrant seeds at 512^2, one octant seed, the Taylor-Green
vortex at step 100; every (cell, axis) pair) sets the logit threshold: the largest that passes at most 0.2 % of the
troubled pairs to the linear reconstruction. Prints the data sizes, the loss per epoch and the held-out figures.
"""
import argparse
import json
import os
import time

import numpy as np

from . import initial
from .runtime import Run
from .sensor import TAU, Sensor, choose_threshold, octant_training_data, quadrant_training_data, taylor_green_training_data

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "sensor_weights.npz")
MISS = 0.002


def held_out(sensor):
    """(features, departures) of every (cell, axis) of the held-out states, by set."""
    torch = sensor.torch
    sets = {}
    Xs, Ds = [], []
    for s in (1000, 1001, 1002, 1003):
        run = Run(initial.quadrant_params(512), U=initial.riemann_quadrants(512, s))
        for t in (0.08, 0.16, 0.25):
            try:
                run.run(t)
            except RuntimeError:
                break
            X, D, _ = sensor.samples(run, mode=0)
            Xs.append(X.clone())
            Ds.append(D.clone())
        run.close()
    sets["quadrants 512^2"] = (torch.cat(Xs), torch.cat(Ds))
    run = Run(initial.octant_params(64), U=initial.riemann_octants(64, 1000))
    Xs, Ds = [], []
    for t in (0.1, 0.2):
        run.run(t)
        X, D, _ = sensor.samples(run, mode=0)
        Xs.append(X.clone())
        Ds.append(D.clone())
    sets["octants 64^3"] = (torch.cat(Xs), torch.cat(Ds))
    import math

    L = 2 * math.pi
    params = dict(nx=64, ny=64, nz=64, Lx=L, Ly=L, Lz=L, gamma=1.4, use_viscous=True, mu=6.25e-4, pr=0.71, riemann_solver="HLLC (Low-Mach Thornber)",
                  reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.5, **{f"bc_{a}{s}": "periodic" for a in "xyz" for s in ("min", "max")})
    run = Run(params, U=initial.taylor_green_3d(64))
    run.run(1e30, max_steps=100)
    X, D, _ = sensor.samples(run, mode=0)
    sets["Taylor-Green 64^3 step 100"] = (X.clone(), D.clone())
    run = Run(dict(params, nx=128, ny=128, nz=128), U=initial.taylor_green_3d(128))
    run.run(1e30, max_steps=6)
    X, D, _ = sensor.samples(run, mode=0)
    sets["Taylor-Green 128^3 step 6"] = (X.clone(), D.clone())
    return sets


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--seeds", type=int, default=64)
    ap.add_argument("--n", type=int, default=512)
    args = ap.parse_args()
    torch = __import__("torch")
    t0 = time.time()
    s = Sensor(seed=0)
    parts = [quadrant_training_data(s, seeds=range(args.seeds), n=args.n, t_end=0.25, snapshots=4, keep_div=16),
             octant_training_data(s, seeds=range(8), n=64, t_end=0.2, snapshots=4, keep_div=16),
             taylor_green_training_data(s, n=64, at=(3, 10, 40, 100, 200), keep_div=4),
             taylor_green_training_data(s, n=128, at=(3, 20), keep_div=4)]
    X = torch.cat([p[0] for p in parts])
    D = torch.cat([p[1] for p in parts])
    del parts
    y = (D > TAU).float()
    print(f"training samples {len(X)} (troubled {y.mean().item():.3f}); data {time.time() - t0:.1f} s", flush=True)
    history = []
    for lr, epochs in ((3e-3, 6), (1e-3, 4), (3e-4, 2)):
        history += s.train(X, y, epochs=epochs, batch=16384, lr=lr)
        print(f"lr {lr}: loss {[round(v, 4) for v in history[-epochs:]]} ({time.time() - t0:.1f} s)", flush=True)
    del X, y, D
    sets = held_out(s)
    zs = {k: s.logits(v[0]) for k, v in sets.items()}
    z_all = torch.cat(list(zs.values()))
    tr_all = torch.cat([v[1] > TAU for v in sets.values()])
    theta = choose_threshold(z_all, tr_all, MISS)
    report = {"tau": TAU, "miss_target": MISS, "threshold": theta, "train_loss": history, "held_out": {}}
    for k, (Xv, Dv) in sets.items():
        z, tr = zs[k], Dv > TAU
        lin = z < theta
        report["held_out"][k] = {"pairs": len(Xv), "troubled": tr.float().mean().item(), "accuracy_at_0": ((z > 0) == tr).float().mean().item(),
                                 "linear_share": lin.float().mean().item(),
                                 "troubled_passed_linear": (lin & tr).float().sum().item() / max(tr.float().sum().item(), 1.0),
                                 "largest_departure_passed": float(Dv[lin].max().item()) if lin.any() else 0.0}
    print(json.dumps(report["held_out"], indent=1), flush=True)
    print(f"threshold {theta:.4f}; total {time.time() - t0:.1f} s")
    s.save(args.out, threshold=np.float32(theta), tau=np.float32(TAU), report=np.array(json.dumps(report)))


if __name__ == "__main__":
    main()
