"""The Mach 2 cylinder configuration and its measures: the bow-shock stand-off distance from a state, and the loads
through Run.ibm_loads (fvg_ibm_loads).

The configuration: an 8 x 12 box, a cylinder of diameter 1 centred at (3, 6) as a sharp ghost-cell immersed boundary
(slip wall), a supersonic inflow rho = 1.4, p = 1, u = 2 sqrt(gamma p / rho) (Mach 2) through a velocity inlet on the left,
transmissive sides elsewhere. The plain form is MUSCL (MC limiter) + HLLC + MUSCL-Hancock, the mixed form WENO5-Z + HLLC +
SSP-RK3.

The stand-off follows the reference's validation measure (cases/validation/verification/ibm_vortex.py:101-113): on
the centre row (the two rows about y = 6, averaged), the first crossing of the density half way between the free
stream and the Mach 2 normal-shock value ((gamma + 1) M^2 / ((gamma - 1) M^2 + 2) = 2.667 times the free stream), upstream
of the body, linearly interpolated; its distance to the body's leading edge over the diameter.
"""
import math

import numpy as np

GAMMA = 1.4
RHO_IN, P_IN, MACH = 1.4, 1.0, 2.0


def cylinder_params(nx=1600, ny=2400, form="plain"):
    u_in = MACH * math.sqrt(GAMMA * P_IN / RHO_IN)
    p = dict(nx=nx, ny=ny, Lx=8.0, Ly=12.0, gamma=GAMMA, riemann_solver="HLLC", cfl=0.5,
             bc_xmin="vel_inlet", bc_xmax="transmissive", bc_ymin="transmissive", bc_ymax="transmissive",
             u_in=u_in, rho_in=RHO_IN, p_out=P_IN, use_ibm=True, ibm_shape="Cylinder", ibm_radius=0.5, ibm_cx=3.0, ibm_cy=6.0)
    if form == "plain":
        p.update(reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock")
    else:
        p.update(reconstruction="weno5", time_scheme="SSP Runge-Kutta 3")
    return p


def free_stream(params):
    """The uniform inflow state on the whole mesh (conservative cells)."""
    n = int(params["nx"]) * int(params["ny"])
    u = float(params["u_in"])
    U = np.zeros((n, 5))
    U[:, 0] = RHO_IN
    U[:, 1] = RHO_IN * u
    U[:, 3] = P_IN / (GAMMA - 1) + 0.5 * RHO_IN * u * u
    return U


def bow_shock_standoff(U, params):
    """Stand-off distance over the diameter, or None without a detected shock."""
    nx, ny = int(params["nx"]), int(params["ny"])
    h = float(params["Lx"]) / nx
    rho = np.asarray(U)[:, 0].reshape(ny, nx)
    row = rho[ny // 2 - 1: ny // 2 + 1].mean(axis=0)
    x = (np.arange(nx) + 0.5) * h
    ratio = (GAMMA + 1) * MACH ** 2 / ((GAMMA - 1) * MACH ** 2 + 2)
    mid = 0.5 * RHO_IN * (1.0 + ratio)
    lead = float(params["ibm_cx"]) - float(params["ibm_radius"])
    found = (row > mid) & (x < lead - 0.5 * h)
    i = int(np.argmax(found))
    if not found.any() or i == 0:
        return None
    xs = x[i - 1] + (mid - row[i - 1]) / (row[i] - row[i - 1]) * h
    return (lead - xs) / (2 * float(params["ibm_radius"]))
