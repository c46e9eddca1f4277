"""The learned troubled-cell sensor: data from WENO5-Z runs, training on the GPU, and the gate of the mixed WENO5-Z form.

The network, its features and its label are described in include/fenice_gpu.h (fvg_sensor_*) and
fenice_b200/csrc/sensor.cuh. This module holds the float32 master parameters, the Adam moments and the device weights in
torch tensors on the GPU (torch provides the device memory and the stream; every computation is a kernel of
libfenice_gpu.so) and drives:

* ``samples(run, tau, keep_div)``: features and label statistics (the largest |WENO5-Z - linear| face-value gap of the
  cell along the axis, relative to the quantity's physical scale) of a run's current state (the troubled (cell, axis)
  pairs and every keep_div-th other one);
* ``train(X, y, ...)``: Adam over minibatches, forward and backward passes on the tensor cores;
* ``logits(X)`` and ``choose_threshold``: the logit below which a cell is passed to the linear reconstruction, chosen so
  that at most a given share of the troubled cells of held-out data is passed (the rest stays WENO5-Z);
* ``Run.set_sensor(sensor, threshold)``: the gate in the stage kernels.
"""
import ctypes

import numpy as np

from . import initial
from .runtime import FVG_OK, Run, load_library

# label: a cell is troubled along an axis when a WENO5-Z face value of it differs from the linear one by more than TAU of
# the quantity's physical scale (the Taylor-Green vortex at 256^3 stays below 2e-7 everywhere; shocks and contacts reach
# 1e-2 to 1)
TAU = 1e-5


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _check(lib, rc, what):
    if rc != FVG_OK:
        raise RuntimeError(f"{what}: {lib.fvg_create_error().decode()}")


class Sensor:
    """The network's parameters on one GPU, trained by the library's kernels."""

    LAYOUT = [("W1", (32, 32)), ("b1", (32,)), ("W2", (32, 32)), ("b2", (32,)), ("w3", (32,)), ("b3", ())]

    def __init__(self, seed=0, device=0, params=None):
        import torch

        self.torch = torch
        self.lib = load_library()
        n_params, n_bytes, n_in = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.fvg_sensor_sizes(ctypes.byref(n_params), ctypes.byref(n_bytes), ctypes.byref(n_in))
        self.n_params, self.n_in = n_params.value, n_in.value
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.current_stream(self.dev)
        if params is None:
            params = self.init_params(seed)
        self.params = torch.tensor(self.flatten(params), dtype=torch.float32, device=self.dev)
        assert self.params.numel() == self.n_params
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad_buf = torch.zeros_like(self.params)
        self.loss_buf = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self.weights = torch.zeros(n_bytes.value, dtype=torch.uint8, device=self.dev)
        self.step = 0
        self.pack()

    # ---- parameters
    @staticmethod
    def init_params(seed):
        """He-normal weights (inputs 25 .. 31 unused), zero biases."""
        rng = np.random.default_rng(seed)
        W1 = rng.normal(0.0, np.sqrt(2.0 / 25), (32, 32))
        W1[:, 25:] = 0.0
        return {"W1": W1, "b1": np.zeros(32), "W2": rng.normal(0.0, np.sqrt(2.0 / 32), (32, 32)), "b2": np.zeros(32),
                "w3": rng.normal(0.0, np.sqrt(1.0 / 32), 32), "b3": 0.0}

    @classmethod
    def flatten(cls, P):
        return np.concatenate([np.asarray(P[k], dtype=np.float32).reshape(-1) for k, _ in cls.LAYOUT])

    @classmethod
    def unflatten(cls, flat):
        out, o = {}, 0
        for k, shape in cls.LAYOUT:
            n = int(np.prod(shape)) if shape else 1
            out[k] = flat[o:o + n].reshape(shape) if shape else float(flat[o])
            o += n
        return out

    def get_params(self):
        return self.unflatten(self.params.cpu().numpy().astype(np.float64))

    def pack(self):
        _check(self.lib, self.lib.fvg_sensor_pack(_p(self.params), _p(self.weights), ctypes.c_void_p(self.stream.cuda_stream)), "sensor_pack")

    def weights_ptr(self):
        return _p(self.weights)

    def save(self, path, **meta):
        np.savez(path, params=self.params.cpu().numpy(), **meta)

    @classmethod
    def load(cls, path, device=0):
        d = np.load(path)
        s = cls(device=device, params=cls.unflatten(d["params"].astype(np.float64)))
        s.meta = {k: d[k] for k in d.files if k != "params"}
        return s

    # ---- data
    def samples(self, run, tau=TAU, keep_div=8, seed=0, capacity=None, mode=1):
        """(X, departure) device tensors of a run's current state: mode 1 the troubled pairs and every keep_div-th other,
        mode 0 every (cell, axis) at index cell * dim + axis."""
        torch = self.torch
        dim = 3 if run.cfg.nz > 1 else 2
        n = run.ncells * dim
        cap = n if (capacity is None or mode == 0) else capacity
        X = torch.empty((cap, self.n_in), dtype=torch.float32, device=self.dev)
        dep = torch.empty(cap, dtype=torch.float32, device=self.dev)
        cnt = torch.zeros(1, dtype=torch.int32, device=self.dev)
        stats = torch.zeros(2, dtype=torch.int64, device=self.dev)
        run.synchronize()
        torch.cuda.synchronize(self.dev)
        _check(self.lib, self.lib.fvg_sensor_extract(run.h, mode, int(keep_div), int(seed) & 0xFFFFFFFF, float(tau), _p(X), _p(dep), _p(cnt), cap,
                                                     _p(stats)), "sensor_extract")
        k = cap if mode == 0 else min(int(cnt.item()), cap)
        return X[:k], dep[:k], stats.cpu().numpy()

    # ---- training
    def grad(self, X, y, wpos=1.0):
        """Loss and gradients (flat float32) of the mean class-weighted cross-entropy over all samples."""
        self.grad_buf.zero_()
        self.loss_buf.zero_()
        _check(self.lib, self.lib.fvg_sensor_grad(_p(self.weights), _p(X), _p(y), len(X), float(wpos), _p(self.grad_buf), _p(self.loss_buf),
                                                  ctypes.c_void_p(self.stream.cuda_stream)), "sensor_grad")
        return float(self.loss_buf.item()) / len(X), self.grad_buf.clone()

    def train(self, X, y, epochs=4, batch=8192, lr=2e-3, wpos=1.0, seed=0):
        """Adam over shuffled minibatches; returns the mean loss of each epoch."""
        torch = self.torch
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(seed)
        out = []
        st = ctypes.c_void_p(self.stream.cuda_stream)
        for _ in range(epochs):
            perm = torch.randperm(len(X), device=self.dev, generator=gen)
            Xs, ys = X[perm].contiguous(), y[perm].contiguous()
            self.loss_buf.zero_()
            for b0 in range(0, len(X), batch):
                nb = min(batch, len(X) - b0)
                self.step += 1
                _check(self.lib, self.lib.fvg_sensor_grad(_p(self.weights), _p(Xs[b0:]), _p(ys[b0:]), nb, float(wpos), _p(self.grad_buf),
                                                          _p(self.loss_buf), st), "sensor_grad")
                _check(self.lib, self.lib.fvg_sensor_adam(_p(self.params), _p(self.m), _p(self.v), _p(self.grad_buf), self.step, float(lr), 0.9,
                                                          0.999, 1e-8, _p(self.weights), st), "sensor_adam")
            out.append(float(self.loss_buf.item()) / len(X))
        return out

    def logits(self, X):
        z = self.torch.empty(len(X), dtype=self.torch.float32, device=self.dev)
        _check(self.lib, self.lib.fvg_sensor_infer(_p(self.weights), _p(X), len(X), _p(z), ctypes.c_void_p(self.stream.cuda_stream)),
               "sensor_infer")
        return z


def choose_threshold(logits, troubled, miss=0.002):
    """The largest logit threshold that passes (logit < threshold) at most `miss` of the troubled samples."""
    z = logits[troubled]
    if z.numel() == 0:
        return 0.0
    k = int(miss * z.numel())
    zs = z.sort().values
    return float(zs[k].item()) if k < zs.numel() else float(zs[-1].item())


def quadrant_training_data(sensor, seeds, n=512, t_end=0.25, snapshots=5, tau=TAU, keep_div=8, precision=0):
    """Samples of seeded four-quadrant problems run with plain WENO5-Z (FP64: the reference's arithmetic), taken at
    `snapshots` evenly spaced times up to t_end (up to the divergence of a problem whose seeded states make WENO5-Z lose
    positivity, as the reference does without its positivity fallback)."""
    torch = sensor.torch
    Xs, Ds = [], []
    for s in seeds:
        run = Run(initial.quadrant_params(n), U=initial.riemann_quadrants(n, s), precision=precision, device=sensor.dev.index)
        for k in range(1, snapshots + 1):
            try:
                run.run(t_end * k / snapshots)
            except RuntimeError:   # the seeded states can make WENO5-Z lose positivity: the snapshots so far stay
                break
            X, D, _ = sensor.samples(run, tau, keep_div, seed=1000 * s + k, capacity=run.ncells * 2)
            Xs.append(X.clone())
            Ds.append(D.clone())
        run.close()
    return torch.cat(Xs), torch.cat(Ds)


def taylor_green_training_data(sensor, n=64, steps=200, snapshots=5, tau=TAU, keep_div=8, precision=0, at=None):
    """Samples of the 3-D Taylor-Green vortex (WENO5-Z + low-Mach HLLC + SSP-RK3, viscous Re 1600) at `snapshots`
    evenly spaced steps, or at the steps listed in `at` (the first steps carry the grid-scale acoustic noise of the
    initial pressure field, of negligible amplitude)."""
    import math

    torch = sensor.torch
    L = 2 * math.pi
    params = dict(nx=n, ny=n, nz=n, Lx=L, Ly=L, Lz=L, gamma=1.4, use_viscous=True, mu=6.25e-4, pr=0.71, riemann_solver="HLLC (Low-Mach Thornber)",
                  reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.5,
                  **{f"bc_{a}{s}": "periodic" for a in "xyz" for s in ("min", "max")})
    run = Run(params, U=initial.taylor_green_3d(n), precision=precision, device=sensor.dev.index)
    Xs, Ds = [], []
    marks = list(at) if at is not None else [steps // snapshots * (k + 1) for k in range(snapshots)]
    done = 0
    for k, mark in enumerate(marks):
        run.run(1e30, max_steps=mark - done)
        done = mark
        X, D, _ = sensor.samples(run, tau, keep_div, seed=77 + k, capacity=run.ncells * 3)
        Xs.append(X.clone())
        Ds.append(D.clone())
    run.close()
    return torch.cat(Xs), torch.cat(Ds)


def octant_training_data(sensor, seeds, n=64, t_end=0.2, snapshots=4, tau=TAU, keep_div=8, precision=0):
    """Samples of seeded eight-octant problems (3-D) run with plain WENO5-Z, as quadrant_training_data."""
    torch = sensor.torch
    Xs, Ds = [], []
    for s in seeds:
        run = Run(initial.octant_params(n), U=initial.riemann_octants(n, s), precision=precision, device=sensor.dev.index)
        for k in range(1, snapshots + 1):
            try:
                run.run(t_end * k / snapshots)
            except RuntimeError:
                break
            X, D, _ = sensor.samples(run, tau, keep_div, seed=5000 + 1000 * s + k, capacity=run.ncells * 3)
            Xs.append(X.clone())
            Ds.append(D.clone())
        run.close()
    return torch.cat(Xs), torch.cat(Ds)
