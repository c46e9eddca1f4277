"""Seeded inputs and the configurations the parity tests run (shared by the tests and tests/golden/make_golden.py).

The fields are smooth random perturbations of a uniform flow (positive density and pressure, every velocity component
non-zero), drawn from numpy's PCG64 with a stated seed, in the reference's layout: cells of 5 doubles
[rho, rho u, rho v, rho E, rho w], cell (k*ny + j)*nx + i; rho w = 0 on a 2-D mesh.
"""
import numpy as np


def prim_to_cons(W, gamma=1.4, p_inf=0.0, stiffened=False):
    """Core.hpp:209-215, elementwise in numpy (IEEE double, the same operation order)."""
    rho, u, v, p, w = W[:, 0], W[:, 1], W[:, 2], W[:, 3], W[:, 4]
    U = np.empty_like(W)
    ke = 0.5 * rho * (u * u + v * v + w * w)
    e = (p + gamma * p_inf) / (gamma - 1.0) if stiffened else p / (gamma - 1.0)
    U[:, 0] = rho
    U[:, 1] = rho * u
    U[:, 2] = rho * v
    U[:, 3] = e + ke
    U[:, 4] = rho * w
    return U


def smooth_field(nx, ny, nz=1, seed=0, amp=0.2, gamma=1.4, jump=False):
    """A seeded field: a few random Fourier modes per variable (plus an optional density / pressure jump)."""
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    x = (i.ravel() + 0.5) / nx
    y = (j.ravel() + 0.5) / ny
    z = (k.ravel() + 0.5) / max(nz, 1)
    W = np.zeros((nx * ny * nz, 5))
    base = [1.0, 0.3, -0.2, 1.0, 0.1 if nz > 1 else 0.0]
    for q in range(5):
        if q == 4 and nz == 1:
            continue
        f = np.full(x.shape, base[q])
        for _ in range(3):
            a, b, c = rng.integers(1, 4, size=3)
            ph = rng.random(3) * 2 * np.pi
            f = f + amp * rng.random() * np.sin(2 * np.pi * a * x + ph[0]) * np.cos(2 * np.pi * b * y + ph[1]) * np.cos(2 * np.pi * c * z + ph[2])
        W[:, q] = f
    if jump:
        left = x < 0.5
        W[left, 0] *= 3.0
        W[left, 3] *= 4.0
    W[:, 0] = np.abs(W[:, 0]) + 0.2
    W[:, 3] = np.abs(W[:, 3]) + 0.2
    return prim_to_cons(W, gamma=gamma)


BC4 = ("bc_xmin", "bc_xmax", "bc_ymin", "bc_ymax")


def bcs(*names, z=("periodic", "periodic")):
    d = dict(zip(BC4, names))
    d["bc_zmin"], d["bc_zmax"] = z
    return d


# residual cases: (name, params, seed, predictor_half_dt)
RESIDUAL_CASES = [
    ("muscl_vl_periodic", dict(nx=24, ny=17, reconstruction="muscl", muscl_limiter="Van Leer", **bcs("periodic", "periodic", "periodic", "periodic")), 1, 0.0),
    ("muscl_minmod_walls", dict(nx=20, ny=19, reconstruction="muscl", muscl_limiter="Minmod", **bcs("wall", "no_slip", "moving_wall", "wall"), u_in=0.3), 2, 0.0),
    ("muscl_mc_inlet", dict(nx=33, ny=16, reconstruction="muscl", muscl_limiter="MC", **bcs("vel_inlet", "transmissive", "transmissive", "outlet"), u_in=1.2, p_out=0.9), 3, 0.0),
    ("muscl_koren_order1", dict(nx=18, ny=31, reconstruction="muscl", muscl_limiter="Koren", boundary_order=1, **bcs("wall", "outlet", "transmissive", "vel_inlet"), v_in=-0.4), 4, 0.0),
    ("weno5_hllc_mixed", dict(nx=35, ny=22, reconstruction="weno5", **bcs("transmissive", "transmissive", "wall", "vel_inlet"), u_in=0.3), 5, 0.0),
    ("weno5_lowmach_periodic", dict(nx=16, ny=30, reconstruction="weno5", riemann_solver="HLLC (Low-Mach Thornber)", **bcs("periodic", "periodic", "periodic", "periodic")), 6, 0.0),
    ("weno3_lowmach_walls", dict(nx=21, ny=18, reconstruction="weno3", riemann_solver="lowmach", **bcs("wall", "outlet", "periodic", "periodic")), 7, 0.0),
    ("weno5_order1_noblend", dict(nx=19, ny=20, reconstruction="weno5", boundary_order=1, shock_blend=0.0, **bcs("no_slip", "transmissive", "wall", "outlet")), 8, 0.0),
    ("first_order_hllc", dict(nx=17, ny=15, reconstruction="none", **bcs("wall", "outlet", "periodic", "periodic")), 9, 0.0),
    ("weno5_stiffened", dict(nx=20, ny=16, reconstruction="weno5", eos_type="Stiffened Gas", gamma=4.4, p_inf=3.0, **bcs("transmissive", "wall", "periodic", "periodic")), 10, 0.0),
    ("weno5_1d_row", dict(nx=64, ny=1, reconstruction="weno5", **bcs("transmissive", "transmissive", "transmissive", "transmissive")), 11, 0.0),
    ("hancock_vl_periodic", dict(nx=24, ny=17, reconstruction="muscl", muscl_limiter="Van Leer", **bcs("periodic", "periodic", "periodic", "periodic")), 12, 0.004),
    ("hancock_mc_inlet", dict(nx=33, ny=18, reconstruction="muscl", muscl_limiter="MC", **bcs("vel_inlet", "transmissive", "wall", "transmissive"), u_in=1.5), 13, 0.003),
    ("hancock_minmod_order1", dict(nx=20, ny=19, reconstruction="muscl", muscl_limiter="Minmod", boundary_order=1, **bcs("no_slip", "outlet", "moving_wall", "wall"), u_in=0.2), 14, 0.005),
    ("w5_3d_periodic_lowmach", dict(nx=12, ny=10, nz=9, reconstruction="weno5", riemann_solver="lowmach", **bcs("periodic", "periodic", "periodic", "periodic")), 15, 0.0),
    ("w5_3d_walls", dict(nx=10, ny=11, nz=12, reconstruction="weno5", **bcs("wall", "transmissive", "no_slip", "vel_inlet", z=("outlet", "wall")), u_in=0.2), 16, 0.0),
    ("muscl_3d_mc", dict(nx=9, ny=12, nz=10, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2", **bcs("transmissive", "outlet", "periodic", "periodic", z=("vel_inlet", "transmissive")), u_in=0.1), 17, 0.0),
    ("visc_3d_periodic", dict(nx=12, ny=9, nz=10, reconstruction="weno5", riemann_solver="lowmach", use_viscous=True, mu=0.02, pr=0.71, **bcs("periodic", "periodic", "periodic", "periodic")), 18, 0.0),
    ("visc_3d_walls", dict(nx=10, ny=9, nz=11, reconstruction="muscl", muscl_limiter="Koren", use_viscous=True, mu=0.01, **bcs("no_slip", "transmissive", "wall", "moving_wall", z=("wall", "wall")), u_in=0.3, v_in=0.1), 19, 0.0),
    ("visc_3d_order1", dict(nx=9, ny=10, nz=8, reconstruction="weno3", boundary_order=1, use_viscous=True, mu=0.01, **bcs("moving_wall", "no_slip", "periodic", "periodic", z=("no_slip", "transmissive")), u_in=0.3, v_in=0.1), 20, 0.0),
]

# time-stepping cases: (name, params, seed, n_steps)
STEP_CASES = [
    ("rk3_weno5_2d", dict(nx=24, ny=20, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4, **bcs("transmissive", "transmissive", "transmissive", "transmissive")), 21, 4),
    ("rk2_muscl_2d", dict(nx=22, ny=18, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2", **bcs("periodic", "periodic", "wall", "wall")), 22, 4),
    ("euler_first_order", dict(nx=20, ny=16, reconstruction="none", time_scheme="Explicit Euler", **bcs("wall", "outlet", "periodic", "periodic")), 23, 5),
    ("hancock_vl_2d", dict(nx=26, ny=21, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="MUSCL-Hancock", **bcs("periodic", "periodic", "periodic", "periodic")), 24, 5),
    ("hancock_mc_inlet", dict(nx=30, ny=20, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock", **bcs("vel_inlet", "transmissive", "transmissive", "wall"), u_in=1.4), 25, 5),
    ("rk3_tgv_like_3d", dict(nx=12, ny=11, nz=10, reconstruction="weno5", riemann_solver="lowmach", time_scheme="SSP Runge-Kutta 3", use_viscous=True, mu=0.01, pr=0.71, **bcs("periodic", "periodic", "periodic", "periodic")), 26, 3),
]


def case_field(params, seed):
    nz = int(params.get("nz", 1))
    gamma = float(params.get("gamma", 1.4))
    U = smooth_field(int(params["nx"]), int(params["ny"]), nz, seed=seed, gamma=gamma, jump=seed % 3 == 0)
    if str(params.get("eos_type", "")).lower().startswith("stiff"):
        W = np.zeros_like(U)
        W[:, 0] = U[:, 0]
        W[:, 1] = U[:, 1] / U[:, 0]
        W[:, 2] = U[:, 2] / U[:, 0]
        W[:, 4] = U[:, 4] / U[:, 0]
        W[:, 3] = 1.0 + 0.1 * np.cos(np.arange(U.shape[0]))
        U = prim_to_cons(W, gamma=gamma, p_inf=float(params["p_inf"]), stiffened=True)
    return U


# immersed-body cases: (name, params, initial primitive state, perturbation seed or None, n_steps)
CYL = dict(Lx=8.0, Ly=12.0, use_ibm=True, ibm_shape="Cylinder", ibm_radius=0.5, ibm_cx=3.0, ibm_cy=6.0, rho_in=1.4, p_out=1.0, u_in=2.0,
           bc_xmin="vel_inlet", bc_xmax="transmissive", bc_ymin="transmissive", bc_ymax="transmissive")
IBM_CASES = [
    ("cyl_hancock_mc", dict(nx=80, ny=120, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock", **CYL), (1.4, 2.0, 0.0, 1.0), 41, 12),
    ("cyl_weno5_rk3", dict(nx=64, ny=96, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.4, **CYL), (1.4, 2.0, 0.0, 1.0), 42, 6),
    ("cyl_minmod_rk2_order1", dict(nx=48, ny=72, reconstruction="muscl", muscl_limiter="Minmod", time_scheme="SSP Runge-Kutta 2",
                                   boundary_order=1, **CYL), (1.4, 2.0, 0.0, 1.0), 43, 6),
    ("sphere3d_weno5_rk3", dict(nx=20, ny=18, nz=22, Lx=1.0, Ly=1.0, Lz=1.0, use_ibm=True, ibm_shape="Sphere", ibm_radius=0.22, ibm_cx=0.45,
                                ibm_cy=0.5, ibm_cz=0.52, rho_in=1.0, p_out=1.0, u_in=0.5, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3",
                                **bcs("vel_inlet", "transmissive", "transmissive", "transmissive", z=("transmissive", "transmissive"))),
     (1.0, 0.5, 0.0, 1.0), 44, 3),
    ("sphere3d_hancock_mc", dict(nx=21, ny=18, nz=19, Lx=1.0, Ly=1.0, Lz=1.0, use_ibm=True, ibm_shape="Sphere", ibm_radius=0.24, ibm_cx=0.45,
                                 ibm_cy=0.5, ibm_cz=0.48, rho_in=1.0, p_out=1.0, u_in=0.6, reconstruction="muscl", muscl_limiter="MC",
                                 time_scheme="MUSCL-Hancock", **bcs("vel_inlet", "transmissive", "wall", "transmissive", z=("periodic", "periodic"))),
     (1.0, 0.6, 0.0, 1.0), 46, 5),
    ("cyl3d_viscous_noslip", dict(nx=24, ny=20, nz=6, Lx=1.2, Ly=1.0, Lz=0.3, use_ibm=True, ibm_shape="Cylinder", ibm_radius=0.2, ibm_cx=0.4,
                                  ibm_cy=0.5, rho_in=1.0, p_out=1.0, u_in=0.4, use_viscous=True, mu=0.01, reconstruction="muscl",
                                  muscl_limiter="Van Leer", time_scheme="SSP Runge-Kutta 2",
                                  **bcs("vel_inlet", "outlet", "wall", "wall", z=("periodic", "periodic"))), (1.0, 0.4, 0.0, 1.0), 45, 3),
]


def ibm_field(params, W0, seed):
    """A uniform primitive state W0 with a small seeded perturbation (cells of 5 doubles; rho w = 0 on a 2-D mesh)."""
    nz = int(params.get("nz", 1))
    U = smooth_field(int(params["nx"]), int(params["ny"]), nz, seed=seed, amp=0.05)
    W = np.zeros_like(U)
    W[:, 0] = W0[0] * U[:, 0]
    W[:, 1] = W0[1] + U[:, 1] / U[:, 0] - 0.3
    W[:, 2] = W0[2] + U[:, 2] / U[:, 0] + 0.2
    W[:, 3] = W0[3] * (1.0 + 0.1 * (U[:, 0] - 1.0))
    if nz > 1:
        W[:, 4] = U[:, 4] / U[:, 0] - 0.1
    return prim_to_cons(W)


# 2-D viscous cases (NavierStokes::viscous_residual_rows): (name, params, seed, steps); a residual of the seeded field,
# then `steps` steps, written by tests/golden/make_golden.py into visc2d.npz
V2 = dict(use_viscous=True, mu=0.02, pr=0.72)
VISC2D_CASES = [
    ("v2_periodic_weno5_rk3", dict(nx=48, ny=40, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", **V2,
                                   **bcs("periodic", "periodic", "periodic", "periodic")), 61, 4),
    ("v2_noslip_muscl_rk2", dict(nx=40, ny=36, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="SSP Runge-Kutta 2", **V2,
                                 **bcs("no_slip", "no_slip", "no_slip", "no_slip")), 62, 4),
    ("v2_lid_weno3_rk3", dict(nx=36, ny=36, reconstruction="weno3", time_scheme="SSP Runge-Kutta 3", u_in=1.0, **V2,
                              **bcs("no_slip", "no_slip", "no_slip", "moving_wall")), 63, 4),
    ("v2_lid_order1", dict(nx=36, ny=34, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", u_in=0.7, v_in=0.2, boundary_order=1, **V2,
                           **bcs("moving_wall", "wall", "no_slip", "moving_wall")), 64, 3),
    ("v2_channel_inlet", dict(nx=50, ny=30, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 3", u_in=0.5, p_out=1.0,
                              **V2, **bcs("vel_inlet", "outlet", "wall", "no_slip")), 65, 4),
    ("v2_xperiodic_walls", dict(nx=44, ny=32, reconstruction="weno5", time_scheme="Explicit Euler", cfl=0.3, **V2,
                                **bcs("periodic", "periodic", "no_slip", "wall")), 66, 3),
    ("v2_yperiodic_first_order", dict(nx=30, ny=40, reconstruction="none", time_scheme="Explicit Euler", **V2,
                                      **bcs("transmissive", "no_slip", "periodic", "periodic")), 67, 3),
]

# 3-D MUSCL-Hancock (MusclReconstruction::hancock_residual_3d): residuals with the predictor of half a step
# (name, params, seed, predictor_half_dt), then steps of the MUSCL-Hancock scheme (name, params, seed, n_steps); sizes that
# leave partial 8 x 8 x 4 tiles, every limiter, periodic, slab and first-order (no halo) sides, walls on every axis
HANCOCK3D_RESIDUAL_CASES = [
    ("h3_vl_periodic", dict(nx=12, ny=10, nz=9, reconstruction="muscl", muscl_limiter="Van Leer", **bcs("periodic", "periodic", "periodic", "periodic")), 31, 0.004),
    ("h3_mc_walls", dict(nx=10, ny=11, nz=7, reconstruction="muscl", muscl_limiter="MC", **bcs("wall", "transmissive", "no_slip", "vel_inlet", z=("outlet", "moving_wall")), u_in=0.3, v_in=-0.2, p_out=0.95), 32, 0.003),
    ("h3_minmod_order1", dict(nx=9, ny=12, nz=10, reconstruction="muscl", muscl_limiter="Minmod", boundary_order=1, **bcs("no_slip", "outlet", "periodic", "periodic", z=("wall", "transmissive"))), 33, 0.005),
    ("h3_koren_lowmach", dict(nx=17, ny=9, nz=6, reconstruction="muscl", muscl_limiter="Koren", riemann_solver="lowmach", **bcs("periodic", "periodic", "wall", "wall", z=("transmissive", "transmissive"))), 34, 0.004),
    ("h3_mc_order1_walls", dict(nx=11, ny=9, nz=13, reconstruction="muscl", muscl_limiter="MC", boundary_order=1, **bcs("moving_wall", "wall", "transmissive", "no_slip", z=("vel_inlet", "outlet")), u_in=0.4), 35, 0.003),
]
HANCOCK3D_STEP_CASES = [
    ("h3s_vl_periodic", dict(nx=12, ny=11, nz=10, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="MUSCL-Hancock", **bcs("periodic", "periodic", "periodic", "periodic")), 36, 5),
    ("h3s_mc_inlet", dict(nx=11, ny=10, nz=9, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock", **bcs("vel_inlet", "transmissive", "wall", "no_slip", z=("periodic", "periodic")), u_in=0.8), 37, 5),
    ("h3s_minmod_order1", dict(nx=10, ny=9, nz=11, reconstruction="muscl", muscl_limiter="Minmod", boundary_order=1, time_scheme="MUSCL-Hancock", **bcs("wall", "outlet", "transmissive", "moving_wall", z=("no_slip", "transmissive")), u_in=0.2), 38, 4),
]

# the body force (ConstantBodyForce) and MUSCL-Hancock with viscous fluxes: a residual (with the predictor of half a step
# for MUSCL-Hancock), then steps; (name, params, seed, predictor_half_dt, n_steps)
FORCE_CASES = [
    ("grav_muscl_rk2_2d", dict(nx=24, ny=20, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2", use_bodyforce=True, gx=0.3,
                               gy=-1.2, **bcs("transmissive", "transmissive", "wall", "wall")), 51, 0.0, 4),
    ("grav_weno5_rk3_3d", dict(nx=10, ny=9, nz=11, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", use_bodyforce=True, gx=-0.2, gy=0.5, gz=-0.9,
                               **bcs("periodic", "periodic", "wall", "no_slip", z=("wall", "transmissive"))), 52, 0.0, 3),
    ("grav_hancock_2d", dict(nx=22, ny=18, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="MUSCL-Hancock", use_bodyforce=True, gx=0.0,
                             gy=-2.0, **bcs("periodic", "periodic", "wall", "wall")), 53, 0.004, 5),
    ("grav_hancock_3d_visc", dict(nx=11, ny=10, nz=9, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock", use_viscous=True, mu=0.02,
                                  use_bodyforce=True, gx=0.4, gy=0.0, gz=-1.5, **bcs("wall", "transmissive", "periodic", "periodic", z=("no_slip", "wall"))),
     54, 0.003, 4),
    ("hancock_visc_2d_walls", dict(nx=20, ny=17, reconstruction="muscl", muscl_limiter="Minmod", time_scheme="MUSCL-Hancock", use_viscous=True, mu=0.03,
                                   **bcs("no_slip", "outlet", "moving_wall", "wall"), u_in=0.3), 55, 0.004, 5),
    ("hancock_visc_3d_order1", dict(nx=9, ny=12, nz=10, reconstruction="muscl", muscl_limiter="Koren", boundary_order=1, time_scheme="MUSCL-Hancock",
                                    use_viscous=True, mu=0.01, riemann_solver="lowmach", **bcs("periodic", "periodic", "no_slip", "moving_wall",
                                                                                                z=("transmissive", "wall")), u_in=0.2), 56, 0.003, 4),
    ("grav_first_order_stiff", dict(nx=30, ny=8, reconstruction="none", time_scheme="Explicit Euler", eos_type="Stiffened Gas", gamma=4.4, p_inf=0.5,
                                    use_bodyforce=True, gx=0.3, gy=-1.0, **bcs("transmissive", "transmissive", "wall", "wall")), 57, 0.0, 6),
    # the mass-flow inlet (its target velocity from the mean density of the side's cells, per residual)
    ("massflow_muscl_rk2_2d", dict(nx=30, ny=16, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2", rho_in=1.2, u_in=0.6,
                                   p_out=0.9, **bcs("massflow_inlet", "outlet", "wall", "wall")), 58, 0.0, 5),
    ("massflow_hancock_order1", dict(nx=28, ny=18, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="MUSCL-Hancock", boundary_order=1,
                                     rho_in=0.9, u_in=0.4, **bcs("massflow_inlet", "transmissive", "periodic", "periodic")), 59, 0.003, 5),
    ("massflow_y_side_2d", dict(nx=20, ny=24, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", rho_in=1.1, u_in=0.3, v_in=0.5,
                                **bcs("wall", "wall", "massflow_inlet", "outlet")), 60, 0.0, 4),
    ("massflow_visc_3d", dict(nx=12, ny=10, nz=9, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", use_viscous=True, mu=0.01, rho_in=1.0,
                              u_in=0.5, **bcs("massflow_inlet", "outlet", "no_slip", "wall", z=("periodic", "periodic"))), 61, 0.0, 3),
    # the non-reflecting outlet (the characteristic ghost with the transverse terms of the side's tangential neighbours:
    # wrapped, one-sided at a wall end, across both other axes in 3-D)
    ("nrbc_muscl_rk2_2d", dict(nx=30, ny=20, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2", p_out=0.95,
                               **bcs("transmissive", "nonreflecting", "periodic", "periodic")), 62, 0.0, 5),
    ("nrbc_hancock_walls_2d", dict(nx=26, ny=18, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="MUSCL-Hancock", u_in=0.5, nrbc_beta=0.3,
                                   **bcs("vel_inlet", "nonreflecting", "wall", "wall")), 63, 0.003, 5),
    ("nrbc_weno5_visc_3d", dict(nx=12, ny=10, nz=9, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", use_viscous=True, mu=0.01, nrbc_sigma=0.5,
                                **bcs("transmissive", "nonreflecting", "no_slip", "wall", z=("nonreflecting", "nonreflecting"))), 64, 0.0, 3),
]


# positivity_fallback (a stage that leaves a cell without density or pressure is repeated with first-order faces around
# it): (name, params, initial state (name, arguments), n_steps). The first two need repairs (the reference diverges
# without the guard); the last two have none (the guarded run has the unguarded bits).
def double_rarefaction(nx, ny, u0, p):
    x = (np.tile(np.arange(nx), ny) + 0.5) / nx
    W = np.zeros((nx * ny, 5))
    W[:, 0] = 1.0
    W[:, 3] = p
    W[:, 1] = np.where(x < 0.5, -u0, u0)
    return prim_to_cons(W)


def blast(nx, ny, nz, p_in, p_out=1e-3):
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    x, y, z = (i.ravel() + 0.5) / nx, (j.ravel() + 0.5) / ny, (k.ravel() + 0.5) / max(nz, 1)
    r2 = (x - 0.5) ** 2 + (y - 0.5) ** 2 + ((z - 0.5) ** 2 if nz > 1 else 0.0)
    W = np.zeros((nx * ny * nz, 5))
    W[:, 0] = 1.0
    W[:, 3] = np.where(r2 < 0.01, p_in, p_out)
    return prim_to_cons(W)


FALLBACK_CASES = [
    ("fb_double_rarefaction_w5", dict(nx=64, ny=4, Ly=1 / 16, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", positivity_fallback=True,
                                      **bcs("transmissive", "transmissive", "periodic", "periodic")), ("double_rarefaction", (64, 4, 3.5, 0.1)), 40),
    ("fb_blast_w5_3d", dict(nx=16, ny=16, nz=16, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.6, positivity_fallback=True,
                            **bcs("periodic", "periodic", "periodic", "periodic")), ("blast", (16, 16, 16, 1e5)), 10),
    ("fb_none_w3_euler", dict(nx=64, ny=4, Ly=1 / 16, reconstruction="weno3", time_scheme="Explicit Euler", cfl=0.3, positivity_fallback=True,
                              **bcs("transmissive", "wall", "periodic", "periodic")), ("double_rarefaction", (64, 4, 2.0, 0.4)), 30),
    ("fb_none_w5_rk3_walls", dict(nx=40, ny=40, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.5, positivity_fallback=True,
                                  **bcs("wall", "wall", "wall", "wall")), ("blast", (40, 40, 1, 1e3)), 12),
]


def fallback_state(spec):
    name, args = spec
    return double_rarefaction(*args) if name == "double_rarefaction" else blast(*args)
