"""Runs with an immersed body in prescribed motion, computed by the reference, for tests/test_gpu_moving.py.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_moving.py

Each case is a case file of ours run by the reference's command-line solver (oracle/_ref/fenice: its own time loop, which
places the body at the start of every step, rebuilds its ghost table when it has moved a quarter cell, fills the cells it
left and checks how far it travelled) for a number of steps, with `dump_state` for the final state. The initial state is
the reference's own set-up of the same case (oracle/ref/ref_harness.cpp, `case` key). A case whose body travels more
than a cell in a step records the reference's error. A section read from a file refers to it as "@section.dat" (its text is
stored in the fixture). tests/golden/moving.npz is test data: nothing of the product reads it.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
FENICE = os.path.join(ROOT, "oracle", "_ref", "fenice")

from oracle.oracle import Reference  # noqa: E402

FLOW2D = """[case]
name = "moving body"
description = "a body moving through a gas at rest with a gentle density gradient"

[initial]
state = { rho = "1.0 + 0.05*x", u = 0.0, v = 0.0, p = "1.0 + 0.02*y" }
"""

FLOW3D = """[case]
name = "moving sphere"
description = "a sphere moving and spinning in a gas"
requires_3d = true

[initial]
state = { rho = "1.0 + 0.05*z", u = 0.1, v = 0.0, w = 0.0, p = 1.0 }
"""

PUSH2D = """[case]
name = "pushed body"
description = "a body in a pressure gradient"

[initial]
state = { rho = "1.0 + 0.1*y", u = 0.05, v = 0.0, p = "1.0 + 0.3*x - 0.1*y" }
"""

PUSH3D = """[case]
name = "pushed sphere"
description = "a sphere in a pressure gradient"
requires_3d = true

[initial]
state = { rho = 1.0, u = 0.0, v = 0.05, w = 0.0, p = "1.0 + 0.2*x + 0.1*z" }
"""

IBM = dict(use_ibm="true", ibm_shape="Cylinder")

STREAM2D = """[case]
name = "airfoil in a stream"
description = "a section in a uniform stream"

[initial]
state = { rho = 1.0, u = 0.5, v = 0.0, p = 1.0 }
"""

STREAM3D = """[case]
name = "extruded airfoil"
description = "an extruded section in a uniform stream"
requires_3d = true

[initial]
state = { rho = 1.0, u = 0.5, v = 0.0, w = 0.0, p = 1.0 }
"""

# a Selig file of our own: a diamond section with a rounded nose, for the file reader (name line, then x y rows)
SECTION_FILE = "diamond-ish section\n" + "\n".join(f"{x:.6f} {y:.6f}" for x, y in (
    (1.0, 0.0), (0.75, 0.03), (0.5, 0.06), (0.25, 0.05), (0.1, 0.035), (0.03, 0.02), (0.0, 0.0), (0.03, -0.02), (0.1, -0.035), (0.25, -0.05),
    (0.5, -0.06), (0.75, -0.03), (1.0, 0.0))) + "\n"
INLET = dict(bc_xmin="vel_inlet", bc_xmax="outlet", bc_ymin="transmissive", bc_ymax="transmissive", u_in=0.5, rho_in=1.0, p_out=1.0)

CASES = {
    "circle_translating_rk2_2d": (FLOW2D, dict(nx=60, ny=40, Lx=3.0, Ly=2.0, reconstruction="muscl", muscl_limiter="Van Leer",
                                               time_scheme="SSP Runge-Kutta 2", bc_xmin="transmissive", bc_xmax="transmissive",
                                               bc_ymin="wall", bc_ymax="wall", ibm_radius=0.3, ibm_cx=1.0, ibm_cy=1.0, ibm_vx=0.4,
                                               ibm_vy=0.1, cfl=0.5, **IBM), 40),
    "circle_spinning_window_viscous_2d": (FLOW2D, dict(nx=40, ny=40, Lx=2.0, Ly=2.0, reconstruction="muscl", muscl_limiter="MC",
                                                       time_scheme="SSP Runge-Kutta 2", use_viscous="true", mu=0.01, bc_xmin="periodic",
                                                       bc_xmax="periodic", bc_ymin="no_slip", bc_ymax="no_slip", ibm_radius=0.35, ibm_cx=1.0,
                                                       ibm_cy=1.0, ibm_omega=3.0, ibm_omega_from=0.02, ibm_omega_until=0.08, ibm_vx=-0.2,
                                                       cfl=0.4, **IBM), 30),
    "circle_hancock_2d": (FLOW2D, dict(nx=50, ny=50, Lx=2.0, Ly=2.0, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock",
                                       bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="transmissive", bc_ymax="transmissive",
                                       ibm_radius=0.25, ibm_cx=1.1, ibm_cy=1.2, ibm_vx=0.3, ibm_vy=-0.5, ibm_omega=-1.0, cfl=0.5, **IBM), 30),
    "sphere_translating_spinning_weno5_3d": (FLOW3D, dict(nx=24, ny=20, nz=20, Lx=1.2, Ly=1.0, Lz=1.0, reconstruction="weno5",
                                                          time_scheme="SSP Runge-Kutta 3", bc_xmin="transmissive", bc_xmax="transmissive",
                                                          bc_ymin="periodic", bc_ymax="periodic", bc_zmin="wall", bc_zmax="wall",
                                                          ibm_shape="Sphere", use_ibm="true", ibm_radius=0.22, ibm_cx=0.5, ibm_cy=0.5, ibm_cz=0.5,
                                                          ibm_vx=0.3, ibm_vz=-0.2, ibm_omega_x=1.5, ibm_omega_y=-0.5, cfl=0.5), 16),
    "sphere_viscous_muscl_3d": (FLOW3D, dict(nx=20, ny=20, nz=16, Lx=1.0, Ly=1.0, Lz=0.8, reconstruction="muscl", muscl_limiter="Van Leer",
                                             time_scheme="SSP Runge-Kutta 2", use_viscous="true", mu=0.005, bc_xmin="transmissive",
                                             bc_xmax="transmissive", bc_ymin="wall", bc_ymax="wall", bc_zmin="periodic", bc_zmax="periodic",
                                             ibm_shape="Sphere", use_ibm="true", ibm_radius=0.2, ibm_cx=0.45, ibm_cy=0.5, ibm_cz=0.4,
                                             ibm_vy=0.25, ibm_omega_y=2.0, cfl=0.4), 16),
    # bodies driven by the flow: the loads of each step's first stage, Adams-Bashforth 2 for the velocities
    "circle_free_rk2_2d": (PUSH2D, dict(nx=60, ny=40, Lx=3.0, Ly=2.0, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="SSP Runge-Kutta 2",
                                        bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="wall", bc_ymax="wall", ibm_radius=0.3,
                                        ibm_cx=1.5, ibm_cy=1.0, ibm_mass=0.2, ibm_vx=0.1, cfl=0.5, **IBM), 40),
    "circle_springs_spin_viscous_2d": (PUSH2D, dict(nx=48, ny=40, Lx=1.2, Ly=1.0, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3",
                                                    use_viscous="true", mu=0.02, bc_xmin="transmissive", bc_xmax="transmissive",
                                                    bc_ymin="no_slip", bc_ymax="no_slip", ibm_radius=0.2, ibm_cx=0.6, ibm_cy=0.5, ibm_mass=0.05,
                                                    ibm_stiff_x=5.0, ibm_damp_y=0.5, ibm_inertia=0.002, ibm_damp_theta=0.001, ibm_omega=0.5,
                                                    cfl=0.4, **IBM), 30),
    "circle_cm_offset_2d": (PUSH2D, dict(nx=50, ny=40, Lx=1.5, Ly=1.2, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2",
                                         use_viscous="true", mu=0.01, bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="wall", bc_ymax="wall",
                                         ibm_radius=0.25, ibm_cx=0.75, ibm_cy=0.6, ibm_mass=0.1, ibm_inertia=0.01, ibm_cm_x=0.05, ibm_cm_y=-0.02,
                                         ibm_stiff_theta=0.5, cfl=0.4, **IBM), 30),
    "sphere_free_3d": (PUSH3D, dict(nx=20, ny=20, nz=20, Lx=1.0, Ly=1.0, Lz=1.0, reconstruction="muscl", muscl_limiter="Van Leer",
                                    time_scheme="SSP Runge-Kutta 3", use_viscous="true", mu=0.01, bc_xmin="transmissive", bc_xmax="transmissive",
                                    bc_ymin="periodic", bc_ymax="periodic", bc_zmin="wall", bc_zmax="wall", ibm_shape="Sphere", use_ibm="true",
                                    ibm_radius=0.2, ibm_cx=0.5, ibm_cy=0.5, ibm_cz=0.5, ibm_mass=0.02, ibm_inertia=0.0005, ibm_stiff_z=2.0,
                                    ibm_damp_theta=0.0001, ibm_omega_x=0.3, cfl=0.5), 14),
    # gravity (the body force): hydrostatic ghost pressures, loads net of the weight, a falling body
    "cylinder_gravity_static_2d": (PUSH2D, dict(nx=40, ny=40, Lx=1.0, Ly=1.0, reconstruction="muscl", muscl_limiter="Van Leer",
                                                time_scheme="MUSCL-Hancock", bc_xmin="wall", bc_xmax="wall", bc_ymin="wall", bc_ymax="wall",
                                                ibm_radius=0.2, ibm_cx=0.5, ibm_cy=0.45, use_bodyforce="true", gx=0.3, gy=-2.0, cfl=0.5, **IBM), 30),
    "circle_falling_viscous_2d": (PUSH2D, dict(nx=40, ny=48, Lx=1.0, Ly=1.2, reconstruction="muscl", muscl_limiter="MC", time_scheme="SSP Runge-Kutta 2",
                                               use_viscous="true", mu=0.01, bc_xmin="no_slip", bc_xmax="no_slip", bc_ymin="wall", bc_ymax="wall",
                                               ibm_radius=0.15, ibm_cx=0.5, ibm_cy=0.7, ibm_mass=0.1, ibm_inertia=0.001, use_bodyforce="true",
                                               gx=0.0, gy=-3.0, cfl=0.4, **IBM), 30),
    "sphere_gravity_weno3_3d": (PUSH3D, dict(nx=18, ny=16, nz=16, Lx=1.0, Ly=1.0, Lz=1.0, reconstruction="weno3", time_scheme="SSP Runge-Kutta 3",
                                             bc_xmin="wall", bc_xmax="wall", bc_ymin="periodic", bc_ymax="periodic", bc_zmin="wall", bc_zmax="wall",
                                             ibm_shape="Sphere", use_ibm="true", ibm_radius=0.2, ibm_cx=0.5, ibm_cy=0.5, ibm_cz=0.55, ibm_mass=0.05,
                                             use_bodyforce="true", gx=0.1, gy=0.0, gz=-1.5, cfl=0.5), 12),
    # sections: NACA 4-digit and a coordinate file, static, pitching, flutter-like, extruded
    "naca0012_static_rk2_2d": (STREAM2D, dict(nx=64, ny=48, Lx=2.0, Ly=1.5, reconstruction="muscl", muscl_limiter="Van Leer",
                                              time_scheme="SSP Runge-Kutta 2", use_ibm="true", ibm_shape="NACA 0012", ibm_chord=0.8, ibm_aoa=5.0,
                                              ibm_cx=0.8, ibm_cy=0.75, cfl=0.5, **INLET), 30),
    "naca2412_pitching_viscous_2d": (STREAM2D, dict(nx=60, ny=50, Lx=1.5, Ly=1.25, reconstruction="muscl", muscl_limiter="MC",
                                                    time_scheme="SSP Runge-Kutta 2", use_viscous="true", mu=0.005, use_ibm="true",
                                                    ibm_shape="NACA2412", ibm_chord=0.6, ibm_aoa=-3.0, ibm_cx=0.6, ibm_cy=0.62, ibm_omega=2.0,
                                                    cfl=0.4, **INLET), 30),
    "section_file_hancock_2d": (STREAM2D, dict(nx=56, ny=40, Lx=1.4, Ly=1.0, reconstruction="muscl", muscl_limiter="MC", time_scheme="MUSCL-Hancock",
                                               use_ibm="true", ibm_shape="Airfoil", ibm_file="@section.dat", ibm_chord=0.7, ibm_aoa=8.0,
                                               ibm_cx=0.55, ibm_cy=0.5, cfl=0.5, **INLET), 25),
    "naca0015_free_pitch_heave_2d": (STREAM2D, dict(nx=60, ny=48, Lx=1.5, Ly=1.2, reconstruction="muscl", muscl_limiter="Van Leer",
                                                    time_scheme="SSP Runge-Kutta 2", use_viscous="true", mu=0.005, use_ibm="true",
                                                    ibm_shape="NACA 0015", ibm_chord=0.5, ibm_aoa=6.0, ibm_cx=0.6, ibm_cy=0.6, ibm_mass=0.05,
                                                    ibm_inertia=0.002, ibm_cm_x=0.05, ibm_cm_y=0.0, ibm_stiff_y=2.0, ibm_stiff_theta=0.05,
                                                    cfl=0.4, **INLET), 30),
    "naca0012_extruded_weno5_3d": (STREAM3D, dict(nx=40, ny=32, nz=4, Lx=1.6, Ly=1.2, Lz=0.2, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3",
                                                  use_ibm="true", ibm_shape="NACA 0012", ibm_chord=0.6, ibm_aoa=4.0, ibm_cx=0.6, ibm_cy=0.6,
                                                  bc_zmin="periodic", bc_zmax="periodic", cfl=0.5, **INLET), 8),
    # the body outruns the ghost table: the reference stops
    "circle_too_fast_2d": (FLOW2D, dict(nx=30, ny=20, Lx=3.0, Ly=2.0, reconstruction="muscl", time_scheme="SSP Runge-Kutta 2",
                                        bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="wall", bc_ymax="wall", ibm_radius=0.3,
                                        ibm_cx=1.0, ibm_cy=1.0, ibm_vx=50.0, cfl=2.5, **IBM), 5),
}


def main():
    out = {}
    tmp = tempfile.mkdtemp(prefix="fvg_moving_")
    section = os.path.join(tmp, "section.dat")
    with open(section, "w") as f:
        f.write(SECTION_FILE)
    for name, (text, params, nsteps) in CASES.items():
        params = {k: (section if v == "@section.dat" else v) for k, v in params.items()}
        case = os.path.join(tmp, name)
        os.makedirs(case)
        path = os.path.join(case, "case.toml")
        with open(path, "w") as f:
            f.write(text)
        U0 = Reference(dict(params, case=path, t_end=1e9)).state()
        dump = os.path.join(case, "final.npz")
        sets = dict(params, t_end=1e9, max_steps=nsteps, save_interval=1000000000, output_root=os.path.join(case, "out"), dump_state=dump)
        cmd = [FENICE, "--case", path, "--no-logo", "--threads", "4"] + sum([["--set", f"{k}={v}"] for k, v in sets.items()], [])
        r = subprocess.run(cmd, capture_output=True, text=True)
        stored = {k: ("@section.dat" if v == section else v) for k, v in dict(params, t_end=1e9).items()}
        out[f"{name}/params"] = np.array(json.dumps(stored))
        out[f"{name}/U0"] = U0
        out[f"{name}/steps"] = np.array(nsteps)
        if r.returncode != 0:
            msg = (r.stderr.strip() or r.stdout.strip()).splitlines()[-1]
            out[f"{name}/error"] = np.array(msg)
            print(f"{name}: the reference stopped: {msg}")
            continue
        with np.load(dump) as z:
            out[f"{name}/U"] = z["U"]
            out[f"{name}/t"] = np.array(float(z["t"]))
            out[f"{name}/step"] = np.array(int(z["step"]))
            print(f"{name}: {int(z['step'])} steps to t = {float(z['t']):.6g}")
    out["file/section.dat"] = np.array(SECTION_FILE)
    np.savez_compressed(os.path.join(HERE, "moving.npz"), **out)


if __name__ == "__main__":
    sys.exit(main())
