"""Residuals and runs with flux_quadrature = fourth computed by the reference, for tests/test_gpu_fourth.py.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_fourth.py

Each case is set up in the reference compiled from its sources (oracle/_ref, through oracle/ref/ref_harness.cpp): the
initial state, its residual and wave speed (Simulation::residual), and the state after a number of steps of the
reference's own time loop with their dt. The cases cover WENO3-Z and WENO5-Z, HLLC and low-Mach HLLC, periodic axes,
sides with and without ghost layers (boundary_order 1 and 2, a non-reflecting outlet), shocks (faces the sensor keeps at
second order), the stiffened gas, the viscous term and the body force. tests/golden/fourth.npz is test data: nothing of
the product reads it.
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Reference  # noqa: E402

RIEMANN2D = """[case]
name = "fourth riemann"
description = "a 2-D Riemann configuration"

[initial]
state = { rho = 0.5313, u = 0.0, v = 0.0, p = 0.4 }

[[initial.region]]
shape = "box"
min = [0.0, 0.0]
max = ["0.5*Lx", "0.5*Ly"]
state = { rho = 0.138, u = 1.206, v = 1.206, p = 0.029 }

[[initial.region]]
shape = "box"
min = ["0.5*Lx", 0.0]
max = ["Lx", "0.5*Ly"]
state = { rho = 0.5323, u = 0.0, v = 1.206, p = 0.3 }

[[initial.region]]
shape = "box"
min = [0.0, "0.5*Ly"]
max = ["0.5*Lx", "Ly"]
state = { rho = 0.5323, u = 1.206, v = 0.0, p = 0.3 }
"""

BLAST3D = """[case]
name = "fourth blast"
description = "a 3-D pressure blob"
requires_3d = true

[initial]
state = { rho = "1.0 + 0.1*x*y", u = 0.05, v = -0.02, w = 0.01, p = 1.0 }

[[initial.region]]
shape = "sphere"
center = ["0.4*Lx", "0.5*Ly", "0.5*Lz"]
radius = "0.2*Lx"
state = { p = 4.0, rho = 1.5 }
"""

WATER = """[case]
name = "fourth water"
description = "a stiffened-gas interface"

[initial]
state = { rho = 1000.0, u = 0.0, v = 0.0, p = 100000.0 }

[[initial.region]]
shape = "cylinder"
center = ["0.5*Lx", "0.5*Ly"]
radius = "0.25*Ly"
state = { rho = 1100.0, p = 300000.0, u = 2.0 }
"""

PER2 = {f"bc_{a}{s}": "periodic" for a in "xy" for s in ("min", "max")}
PER3 = {f"bc_{a}{s}": "periodic" for a in "xyz" for s in ("min", "max")}

CASES = {
    "vortex_weno5_rk3_2d": (dict(nx=32, ny=32, Lx=10.0, Ly=10.0, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", flux_quadrature="fourth",
                                 t_end=1e9, **PER2), {"initial_profile": "isentropic_vortex"}, 12),
    "riemann_weno3_b1_2d": (dict(nx=40, ny=40, reconstruction="weno3", time_scheme="SSP Runge-Kutta 3", flux_quadrature="fourth", boundary_order=1,
                                 bc_xmin="wall", bc_xmax="transmissive", bc_ymin="no_slip", bc_ymax="transmissive", t_end=1e9), RIEMANN2D, 10),
    "riemann_weno5_b2_lowmach_euler_2d": (dict(nx=36, ny=30, reconstruction="weno5", time_scheme="Explicit Euler", flux_quadrature="fourth",
                                                riemann_solver="HLLC (Low-Mach Thornber)", boundary_order=2, bc_xmin="transmissive",
                                                bc_xmax="outlet", bc_ymin="wall", bc_ymax="vel_inlet", u_in=0.1, v_in=-0.3, p_out=0.35,
                                                use_bodyforce="true", gx=0.1, gy=-0.5, cfl=0.3, t_end=1e9), RIEMANN2D, 8),
    "water_weno3_stiffened_2d": (dict(nx=32, ny=24, Lx=1.0, Ly=0.75, reconstruction="weno3", time_scheme="SSP Runge-Kutta 3", flux_quadrature="fourth",
                                      eos_type="Stiffened Gas", gamma=4.4, p_inf=6.0e8, bc_xmin="transmissive", bc_xmax="transmissive",
                                      bc_ymin="periodic", bc_ymax="periodic", t_end=1e9), WATER, 6),
    "tgv_weno5_rk3_viscous_3d": (dict(nx=12, ny=10, nz=8, Lx=6.283185307179586, Ly=6.283185307179586, Lz=6.283185307179586, reconstruction="weno5",
                                      time_scheme="SSP Runge-Kutta 3", flux_quadrature="fourth", riemann_solver="HLLC (Low-Mach Thornber)",
                                      use_viscous="true", mu=0.01, t_end=1e9, **PER3), {"initial_profile": "taylor_green_3d"}, 5),
    "blast_weno5_walls_nrbc_3d": (dict(nx=14, ny=10, nz=9, Lx=1.4, Ly=1.0, Lz=0.9, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3",
                                       flux_quadrature="fourth", boundary_order=2, bc_xmin="wall", bc_xmax="nonreflecting", bc_ymin="periodic",
                                       bc_ymax="periodic", bc_zmin="no_slip", bc_zmax="transmissive", p_out=1.0, t_end=1e9), BLAST3D, 6),
    "blast_weno3_b1_3d": (dict(nx=10, ny=9, nz=8, Lx=1.0, Ly=0.9, Lz=0.8, reconstruction="weno3", time_scheme="SSP Runge-Kutta 3", flux_quadrature="fourth",
                               boundary_order=1, bc_xmin="transmissive", bc_xmax="outlet", bc_ymin="wall", bc_ymax="wall", bc_zmin="periodic",
                               bc_zmax="periodic", p_out=1.0, t_end=1e9), BLAST3D, 6),
}


def main():
    out = {}
    tmp = tempfile.mkdtemp(prefix="fvg_fourth_")
    for name, (params, init, nsteps) in CASES.items():
        if isinstance(init, str):
            path = os.path.join(tmp, f"{name}.toml")
            with open(path, "w") as f:
                f.write(init)
            ref = Reference(dict(params, case=path))
        else:
            ref = Reference(params, **init)
        U0 = ref.state()
        R, s = ref.residual(U0)
        ref.set_state(U0)
        ref.t = 0.0
        dts, _ = ref.steps(nsteps, float(params["t_end"]))
        out[f"{name}/params"] = np.array(json.dumps(params))
        out[f"{name}/U0"] = U0
        out[f"{name}/R"] = R
        out[f"{name}/s"] = np.array(s)
        out[f"{name}/dts"] = dts
        out[f"{name}/U"] = ref.state()
        out[f"{name}/t"] = np.array(ref.t)
        print(f"{name}: residual speed {s:.6g}, {len(dts)} steps to t = {ref.t:.6g}")
    np.savez_compressed(os.path.join(HERE, "fourth.npz"), **out)


if __name__ == "__main__":
    sys.exit(main())
