"""Checkpoints written by the reference, and the state its uninterrupted run reaches, for the checkpoint interop tests.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_checkpoint.py

For each case below (a case file of ours: a 2-D diaphragm problem run with MUSCL-Hancock, whose checkpoint carries the
lagged wave speed S; a 3-D viscous periodic box run with WENO5-Z and SSP-RK3; immersed bodies whose checkpoints carry
body_pose: a 2-D circle driven by the flow on springs with a driven rotation, a 3-D sphere in prescribed translation and
spin, a 3-D sphere driven by the flow with a driven rotation), the reference command-line solver
(oracle/_ref/fenice) is run
  1. for STOP steps: its checkpoint (<output>/<case>/<case>_restart.npz) is copied byte for byte to tests/golden/ckpt_<name>.npz;
  2. for TOTAL steps without interruption, with dump_state: the final state;
  3. resumed (resume = true) from the checkpoint of 1 for TOTAL - STOP steps, with dump_state: it must equal 2 bit for bit
     (the reference's own restart is exact).
tests/golden/ckpt_final.npz holds, per case, the resolved parameters (`fenice --print-config`), the case file, the final
state of 2, its time and step count, the --set keys of the case, and where the reference looks for its checkpoint under
output_root. The fixtures are test data: nothing of the product reads them.
"""
import glob
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
FENICE = os.path.join(ROOT, "oracle", "_ref", "fenice")
STOP, TOTAL = 7, 15

DIAPHRAGM = """[case]
name = "ckpt_diaphragm"
description = "a diaphragm problem for the checkpoint interop tests"

[initial]
state = { rho = 0.125, u = 0.0, v = 0.0, p = 0.1 }

[[initial.region]]
shape = "halfspace"
point = ["0.4*Lx", 0.0]
normal = [-1.0, 0.0]
state = { rho = 1.0, u = 0.3, p = 1.0 }
"""

BOX = """[case]
name = "ckpt_box"
description = "a viscous periodic box for the checkpoint interop tests"

[initial]
state = { rho = "1.0 + 0.1*sin(x)*cos(z)", u = "sin(x)*cos(y)*cos(z)", v = "-cos(x)*sin(y)*cos(z)", w = "0.2*sin(z)", p = "100.0 + 0.0625*(cos(2*x) + cos(2*y))*(cos(2*z) + 2.0)" }
"""

PUSH2D = """[case]
name = "ckpt_pushed_body"
description = "a body in a pressure gradient, for the checkpoint interop tests"

[initial]
state = { rho = "1.0 + 0.1*y", u = 0.05, v = 0.0, p = "1.0 + 0.3*x - 0.1*y" }
"""

PUSH3D = """[case]
name = "ckpt_pushed_sphere"
description = "a sphere in a pressure gradient, for the checkpoint interop tests"
requires_3d = true

[initial]
state = { rho = 1.0, u = 0.0, v = 0.05, w = 0.0, p = "1.0 + 0.2*x + 0.1*z" }
"""

CASES = {
    "hancock_2d": (DIAPHRAGM, dict(nx=60, ny=10, Lx=1.0, Ly=0.1, reconstruction="muscl", muscl_limiter="Van Leer", time_scheme="MUSCL-Hancock",
                                   bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="wall", bc_ymax="wall", boundary_order=1)),
    "weno5_rk3_3d": (BOX, dict(nx=12, ny=10, nz=8, Lx=6.283185307179586, Ly=6.283185307179586, Lz=6.283185307179586, reconstruction="weno5",
                               time_scheme="SSP Runge-Kutta 3", riemann_solver="HLLC (Low-Mach Thornber)", use_viscous="true", mu=0.01, cfl=0.5,
                               **{f"bc_{a}{s}": "periodic" for a in "xyz" for s in ("min", "max")})),
    "free_circle_rk2_2d": (PUSH2D, dict(nx=48, ny=40, Lx=1.2, Ly=1.0, reconstruction="muscl", muscl_limiter="Van Leer",
                                        time_scheme="SSP Runge-Kutta 2", bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="wall",
                                        bc_ymax="wall", use_ibm="true", ibm_shape="Cylinder", ibm_radius=0.2, ibm_cx=0.6, ibm_cy=0.5,
                                        ibm_mass=0.05, ibm_stiff_x=5.0, ibm_inertia=0.002, ibm_damp_theta=0.001, ibm_omega=0.5, ibm_vx=0.2,
                                        cfl=0.5)),
    "prescribed_sphere_3d": (PUSH3D, dict(nx=16, ny=16, nz=16, Lx=1.0, Ly=1.0, Lz=1.0, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3",
                                          bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="periodic", bc_ymax="periodic",
                                          bc_zmin="wall", bc_zmax="wall", use_ibm="true", ibm_shape="Sphere", ibm_radius=0.2, ibm_cx=0.5,
                                          ibm_cy=0.5, ibm_cz=0.5, ibm_vx=0.6, ibm_vz=-0.3, ibm_omega_x=1.5, cfl=0.5)),
    "free_sphere_3d": (PUSH3D, dict(nx=16, ny=16, nz=16, Lx=1.0, Ly=1.0, Lz=1.0, reconstruction="muscl", muscl_limiter="MC",
                                    time_scheme="SSP Runge-Kutta 3", bc_xmin="transmissive", bc_xmax="transmissive", bc_ymin="periodic",
                                    bc_ymax="periodic", bc_zmin="wall", bc_zmax="wall", use_ibm="true", ibm_shape="Sphere", ibm_radius=0.2,
                                    ibm_cx=0.5, ibm_cy=0.5, ibm_cz=0.5, ibm_mass=0.02, ibm_inertia=0.0005, ibm_stiff_z=2.0,
                                    ibm_damp_theta=0.0001, ibm_omega_x=0.3, ibm_vy=0.2, cfl=0.5)),
}


def run(case_dir, sets, extra):
    cmd = [FENICE, "--case", os.path.join(case_dir, "case.toml"), "--no-logo", "--threads", "2"]
    for k, v in dict(sets, **extra).items():
        cmd += ["--set", f"{k}={v}"]
    return subprocess.run(cmd, capture_output=True, text=True, check=True).stdout


def resolved(case_dir, sets):
    out = subprocess.run([FENICE, "--case", os.path.join(case_dir, "case.toml"), "--no-logo", "--print-config"] +
                         sum([["--set", f"{k}={v}"] for k, v in sets.items()], []), capture_output=True, text=True, check=True).stdout
    return {k.strip(): v.strip() for k, v in (line.split(" = ", 1) for line in out.splitlines() if " = " in line)}


def main():
    final = {}
    for name, (text, sets) in CASES.items():
        tmp = tempfile.mkdtemp(prefix="fvg_ckpt_")
        with open(os.path.join(tmp, "case.toml"), "w") as f:
            f.write(text)
        sets = dict(sets, t_end=1e9, save_interval=1000000000)
        out1 = os.path.join(tmp, "out1")
        run(tmp, sets, {"max_steps": STOP, "output_root": out1})
        ck = glob.glob(os.path.join(out1, "**", "*_restart.npz"), recursive=True)
        assert len(ck) == 1, ck
        shutil.copyfile(ck[0], os.path.join(HERE, f"ckpt_{name}.npz"))
        run(tmp, sets, {"max_steps": TOTAL, "output_root": os.path.join(tmp, "out2"), "dump_state": os.path.join(tmp, "whole.npz")})
        # (a resumed run counts max_steps from where it resumes)
        run(tmp, sets, {"max_steps": TOTAL - STOP, "output_root": out1, "resume": "true", "dump_state": os.path.join(tmp, "resumed.npz")})
        whole, resumed = np.load(os.path.join(tmp, "whole.npz")), np.load(os.path.join(tmp, "resumed.npz"))
        same = np.array_equal(whole["U"].view(np.uint64), resumed["U"].view(np.uint64)) and int(whole["step"]) == int(resumed["step"])
        print(f"{name}: checkpoint at step {int(np.load(os.path.join(HERE, f'ckpt_{name}.npz'))['step'])}, whole run {int(whole['step'])} steps to t = {float(whole['t']):.6g}; "
              f"the reference resumed from its checkpoint {'equals' if same else 'DIFFERS FROM'} its whole run")
        final[f"{name}/params"] = np.array(json.dumps(resolved(tmp, sets)))
        final[f"{name}/sets"] = np.array(json.dumps({k: str(v) for k, v in sets.items()}))
        final[f"{name}/case_toml"] = np.array(text)
        final[f"{name}/U"] = whole["U"]
        final[f"{name}/t"] = np.array(float(whole["t"]))
        final[f"{name}/step"] = np.array(int(whole["step"]))
        final[f"{name}/resume_exact"] = np.array(same)
        final[f"{name}/ckpt_relpath"] = np.array(os.path.relpath(ck[0], out1))
        shutil.rmtree(tmp, ignore_errors=True)
    np.savez_compressed(os.path.join(HERE, "ckpt_final.npz"), **final)


if __name__ == "__main__":
    sys.exit(main())
