"""Initial states of the benchmark configurations, as conservative cells [rho, rho u, rho v, rho E, rho w] in the
reference's cell order ((k ny + j) nx + i), evaluated at cell centres.

* ``taylor_green_3d``: the compressible Taylor-Green vortex (the reference's taylor_green_3d profile,
  cpp/src/TestCases.cpp:264-271).
* ``riemann_quadrants``: four constant states split at (0.5, 0.5) of [0,1]^2, drawn from a seeded PCG64 in NE, NW, SW,
  SE order with rho, p ~ U[0.1, 2], u, v ~ U[-1, 1] (a case file with a background state and three box regions,
  CaseFile.hpp:110-111, describes the same field).
* ``riemann_octants``: the 3-D analogue, eight constant states split at (0.5, 0.5, 0.5) of [0,1]^3 (training data of
  the learned sensor).
* ``shock_tubes``: a batch of seeded 1-D shock tubes on nx x 1 meshes, nx log-uniform in [128, 8192], interface at
  x = 0.5, rho ~ U[0.1, 1], p ~ U[0.05, 1], u ~ U[-1, 1] on each side.
"""
import math

import numpy as np


def prim_to_cons(W, gamma=1.4):
    """Conservative cells of primitive cells [rho, u, v, p, w] (ideal gas; EOS::prim_to_cons, cpp/include/fv/Core.hpp:209-221)."""
    W = np.asarray(W, dtype=np.float64)
    U = np.empty_like(W)
    r, u, v, p, w = W[:, 0], W[:, 1], W[:, 2], W[:, 3], W[:, 4]
    U[:, 0] = r
    U[:, 1] = r * u
    U[:, 2] = r * v
    U[:, 3] = p / (gamma - 1.0) + 0.5 * r * (u * u + v * v + w * w)
    U[:, 4] = r * w
    return U


def taylor_green_3d(n, gamma=1.4, mach=0.1):
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0, rho = 1, p = 1/(gamma Ma^2) + (cos 2x + cos 2y)(cos 2z + 2)/16 on
    n^3 cells of [0, 2 pi]^3."""
    h = 2 * math.pi / n
    c = (np.arange(n) + 0.5) * h
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    u = (np.sin(x) * np.cos(y) * np.cos(z)).ravel()
    v = (-np.cos(x) * np.sin(y) * np.cos(z)).ravel()
    p = (1.0 / (gamma * mach * mach) + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0).ravel()
    U = np.zeros((n ** 3, 5))
    U[:, 0] = 1.0
    U[:, 1] = u
    U[:, 2] = v
    U[:, 3] = p / (gamma - 1.0) + 0.5 * (u * u + v * v)
    return U


def quadrant_states(seed):
    """The four (rho, u, v, p) states of a seeded four-quadrant problem, NE, NW, SW, SE."""
    rng = np.random.default_rng(seed)
    return [(rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.1, 2)) for _ in range(4)]


def riemann_quadrants(n, seed, gamma=1.4):
    """The seeded four-quadrant Riemann problem on n x n cells of [0, 1]^2."""
    st = quadrant_states(seed)
    c = (np.arange(n) + 0.5) / n
    y, x = np.meshgrid(c, c, indexing="ij")
    x, y = x.ravel(), y.ravel()
    q = np.where(x >= 0.5, np.where(y >= 0.5, 0, 3), np.where(y >= 0.5, 1, 2))
    W = np.zeros((n * n, 5))
    for k, (r, u, v, p) in enumerate(st):
        W[q == k] = (r, u, v, p, 0.0)
    return prim_to_cons(W, gamma)


def quadrant_params(n):
    """WENO5-Z + HLLC + SSP-RK3, CFL 0.4, transmissive sides, [0, 1]^2 (run to t = 0.25)."""
    return dict(nx=n, ny=n, Lx=1.0, Ly=1.0, gamma=1.4, reconstruction="weno5", riemann_solver="HLLC", time_scheme="SSP Runge-Kutta 3",
                cfl=0.4, bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="transmissive", bc_ymax="transmissive")


def riemann_octants(n, seed, gamma=1.4):
    """Eight constant states (rho, p ~ U[0.1, 2], u, v, w ~ U[-1, 1], drawn in octant order x fastest) on n^3 cells of
    [0, 1]^3."""
    rng = np.random.default_rng(seed)
    st = [(rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.1, 2), rng.uniform(-1, 1)) for _ in range(8)]
    c = (np.arange(n) + 0.5) / n
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    o = ((x >= 0.5).astype(int) + 2 * (y >= 0.5) + 4 * (z >= 0.5)).ravel()
    W = np.zeros((n ** 3, 5))
    for k, w in enumerate(st):
        W[o == k] = w
    return prim_to_cons(W, gamma)


def octant_params(n):
    """WENO5-Z + HLLC + SSP-RK3, CFL 0.4, transmissive sides, [0, 1]^3."""
    p = dict(quadrant_params(n), nz=n, Lz=1.0, bc_zmin="transmissive", bc_zmax="transmissive")
    return p


def shock_tubes(n=512, seed=0, nx_min=128, nx_max=8192, gamma=1.4):
    """A batch of n seeded shock tubes: (parameter dicts, conservative states, left / right primitive states (rho, u, p)).
    Each problem is nx x 1 cells of [0, 1] x [0, 1/nx] (square cells), WENO5-Z + HLLC + SSP-RK3, CFL 0.4, transmissive sides,
    to be run to t = 0.15."""
    rng = np.random.default_rng(seed)
    nxs = np.rint(np.exp(rng.uniform(math.log(nx_min), math.log(nx_max), n))).astype(int)
    params, states, lr = [], [], []
    for nx in nxs:
        left = (rng.uniform(0.1, 1.0), rng.uniform(-1.0, 1.0), rng.uniform(0.05, 1.0))
        right = (rng.uniform(0.1, 1.0), rng.uniform(-1.0, 1.0), rng.uniform(0.05, 1.0))
        nx = int(nx)
        params.append(dict(nx=nx, ny=1, Lx=1.0, Ly=1.0 / nx, gamma=gamma, reconstruction="weno5", riemann_solver="HLLC",
                           time_scheme="SSP Runge-Kutta 3", cfl=0.4, bc_xmin="transmissive", bc_xmax="transmissive",
                           bc_ymin="transmissive", bc_ymax="transmissive"))
        xc = (np.arange(nx) + 0.5) / nx
        W = np.zeros((nx, 5))
        on_left = xc < 0.5
        W[on_left, 0], W[on_left, 1], W[on_left, 3] = left
        W[~on_left, 0], W[~on_left, 1], W[~on_left, 3] = right
        states.append(prim_to_cons(W, gamma))
        lr.append((left, right))
    return params, states, lr
