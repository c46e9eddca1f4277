"""Runs with case-file source terms and time-dependent boundary values, computed by the reference, for
tests/test_gpu_sources.py.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_sources.py

Each case below is set up in the reference compiled from its sources (oracle/_ref, through oracle/ref/ref_harness.cpp):
its initial state, its residual of that state at a few stage times (Simulation::residual with the scheme's stage_time,
and for MUSCL-Hancock its predictor of half a step), and the state after a number of steps of its own time loop with
their dt. A case whose boundary value stops being positive is recorded with the reference's error. The time tables are
written next to the fixture as text and stored in it. tests/golden/sources.npz is test data: nothing of the product
reads it.
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Reference  # noqa: E402

PERIODIC3 = {f"bc_{a}{s}": "periodic" for a in "xyz" for s in ("min", "max")}
PERIODIC2 = {f"bc_{a}{s}": "periodic" for a in "xy" for s in ("min", "max")}

SRC_STEADY3 = dict(source_rho="0.05*sin(2*pi*x/Lx)*cos(2*pi*z/Lz)", source_mx="0.1*cos(2*pi*y/Ly) + mu*x",
                   source_my="-0.1*sin(2*pi*x/Lx)*exp(-z)", source_E="0.2*(1 + 0.5*cos(2*pi*(x + y)/Lx))", source_mz="0.03*y*z - 0.01")
SRC_UNSTEADY2 = dict(source_rho="0.1*pi*cos(pi*(x + y - t))*(1 + 0.2*sin(pi*x))", source_mx="0.2*sin(2*pi*x - 3*t)",
                     source_my="0.05*cos(2*pi*y + t)*exp(-t)", source_E="0.3*sin(pi*x)*sin(pi*y)*cos(5*t) + 0.01*t")
SRC_UNSTEADY3 = dict(source_rho="0.02*sin(2*pi*(x - t))", source_mx="0.05*cos(2*pi*z + 2*t)", source_my="0.01*t*y",
                     source_E="0.1*sin(2*pi*x)*cos(2*pi*y)*sin(3*t + z)", source_mz="-0.04*sin(2*pi*y - t)")

TABLES = {
    "inlet_u.csv": "t,value\n0.0, 0.4\n0.01, 0.55\n0.02, 0.5\n0.05, 0.6\n",
    "inlet_v.csv": "# tangential inflow\n0 0.0\n0.015 0.05\n1 0.05\n",
    "outlet_p.csv": "0.0,0.9\n0.02,0.85\n0.04,0.95\n",
    "massflow_rho.csv": "0,1.0\n0.005,1.1\n0.03,1.25\n",
}

CASES = {
    # steady sources: evaluated once, on the host with the C library's functions (the reference's bits)
    "steady_weno5_rk3_3d": (dict(nx=12, ny=10, nz=8, Lx=1.0, Ly=1.0, Lz=1.0, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3",
                                 riemann_solver="HLLC (Low-Mach Thornber)", use_viscous="true", mu=0.01, cfl=0.5, t_end=1.0, **PERIODIC3,
                                 **SRC_STEADY3), {"initial_profile": "taylor_green_3d"}, 6, (0.0, 0.02)),
    "steady_hancock_bodyforce_2d": (dict(nx=30, ny=20, Lx=1.5, Ly=1.0, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock",
                                         bc_xmin="wall", bc_xmax="wall", bc_ymin="no_slip", bc_ymax="wall", use_bodyforce="true", gx=0.3, gy=-1.0,
                                         source_rho="0.01*x*y", source_mx="0.02*sin(3*x)", source_my="-0.05*y^2", source_E="0.1*cos(pi*x)*y",
                                         t_end=1.0), {"initial_profile": "isentropic_vortex"}, 8, (0.0, 0.01)),
    # unsteady sources: evaluated on the device at every stage time (CUDA's functions)
    "unsteady_muscl_rk3_2d": (dict(nx=24, ny=20, Lx=1.0, Ly=1.0, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="SSP Runge-Kutta 3",
                                   t_end=1.0, **PERIODIC2, **SRC_UNSTEADY2), {"initial_profile": "isentropic_vortex"}, 10, (0.0, 0.013, 0.5)),
    "unsteady_hancock_3d": (dict(nx=10, ny=8, nz=8, Lx=1.0, Ly=1.0, Lz=1.0, reconstruction="muscl", muscl_limiter="Minmod", time_scheme="MUSCL-Hancock",
                                 t_end=1.0, **PERIODIC3, **SRC_UNSTEADY3), {"initial_profile": "taylor_green_3d"}, 7, (0.0, 0.021)),
    # boundary values from time tables (arithmetic only: the reference's bits)
    "table_inlet_outlet_rk2_2d": (dict(nx=40, ny=12, Lx=2.0, Ly=0.6, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="SSP Runge-Kutta 2",
                                       bc_xmin="vel_inlet", bc_xmax="outlet", bc_ymin="wall", bc_ymax="wall", u_in_table="inlet_u.csv",
                                       v_in_table="inlet_v.csv", p_out_table="outlet_p.csv", t_end=1.0), {"initial_state": (1.0, 0.4, 0.0, 0.9)}, 25,
                                  (0.0, 0.004, 0.0125, 0.3)),
    # boundary values as expressions of t: arithmetic ones (the reference's bits), the mass-flow inlet's density from a table
    "expr_massflow_weno3_2d": (dict(nx=36, ny=10, Lx=1.2, Ly=0.4, reconstruction="weno3", time_scheme="SSP Runge-Kutta 3", bc_xmin="massflow_inlet",
                                    bc_xmax="outlet", bc_ymin="wall", bc_ymax="wall", u_in="0.3 + 5*t", v_in="0.02*t", rho_in_table="massflow_rho.csv",
                                    p_out="1 - 2*t*t", t_end=1.0), {"initial_state": (1.0, 0.3, 0.0, 1.0)}, 20, (0.0, 0.01, 0.02)),
    # a moving wall whose speed is a transcendental expression of t, viscous (CUDA's sin on the device)
    "expr_moving_wall_viscous_2d": (dict(nx=20, ny=20, Lx=1.0, Ly=1.0, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="SSP Runge-Kutta 2",
                                         bc_xmin="periodic", bc_xmax="periodic", bc_ymin="no_slip", bc_ymax="moving_wall", u_in="0.5*sin(40*t)",
                                         use_viscous="true", mu=0.02, t_end=1.0), {"initial_state": (1.0, 0.0, 0.0, 1.0)}, 20, (0.0, 0.01)),
    # p_out falls below zero: the reference stops with an error
    "falling_p_out_rk3_2d": (dict(nx=20, ny=8, Lx=1.0, Ly=0.4, reconstruction="muscl", time_scheme="SSP Runge-Kutta 3", bc_xmin="transmissive",
                                  bc_xmax="outlet", bc_ymin="wall", bc_ymax="wall", p_out="1 - 40*t", t_end=1.0), {"initial_state": (1.0, 0.1, 0.0, 1.0)},
                             200, ()),
}


def main():
    tmp = tempfile.mkdtemp(prefix="fvg_src_")
    for name, text in TABLES.items():
        with open(os.path.join(tmp, name), "w") as f:
            f.write(text)
    out = {}
    for name, (params, init, nsteps, stage_times) in CASES.items():
        p = {k: (os.path.join(tmp, v) if k.endswith("_table") else v) for k, v in params.items()}
        ref = Reference(p, **init)
        U0 = ref.state()
        out[f"{name}/params"] = np.array(json.dumps(params))
        out[f"{name}/U0"] = U0
        hancock = params.get("time_scheme") == "MUSCL-Hancock"
        for i, st in enumerate(stage_times):
            R, s = ref.residual(U0, stage_time=st)
            out[f"{name}/R{i}"] = R
            out[f"{name}/s{i}"] = np.array(s)
            if hancock:
                Rh, sh = ref.residual(U0, stage_time=st + 0.004, predictor_half_dt=0.004)
                out[f"{name}/Rh{i}"] = Rh
                out[f"{name}/sh{i}"] = np.array(sh)
        out[f"{name}/stage_times"] = np.array(stage_times, dtype=np.float64)
        ref.set_state(U0)
        ref.t = 0.0
        try:
            dts, _ = ref.steps(nsteps, float(params["t_end"]))
            out[f"{name}/dts"] = dts
            out[f"{name}/U"] = ref.state()
            out[f"{name}/t"] = np.array(ref.t)
            print(f"{name}: {len(dts)} steps to t = {ref.t:.6g}")
        except RuntimeError as e:
            out[f"{name}/error"] = np.array(str(e))
            print(f"{name}: the reference stopped: {e}")
    for tname, text in TABLES.items():
        out[f"table/{tname}"] = np.array(text)
    np.savez_compressed(os.path.join(HERE, "sources.npz"), **out)


if __name__ == "__main__":
    sys.exit(main())
