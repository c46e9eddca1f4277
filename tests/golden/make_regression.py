"""The reference's own regression fixtures for the uniform-mesh path, with the inputs the parity tests need.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_regression.py /path/to/fenice

The reference keeps the final states of short runs (cpp/tests/reference/<case>.npz: U, step) and checks its solver
against them in cpp/tests/regression.py (relative difference per variable, against that variable's largest magnitude,
below 1e-8). For the cases named in CASES (the uniform-mesh ones: no AMR, MPI strips or hot start), this script takes
the case's entry of the reference's own table (regression.py's CASES: a test case and overrides; the module is imported
from the reference tree, with FENICE_EXE pointing at oracle/_ref/fenice) and writes tests/golden/regression.npz:

  <case>/params    the resolved parameters (`fenice --print-config` with the options regression.py runs the case with;
                   JSON of strings)
  <case>/U0        the initial state the reference sets up (Simulation::initialize_field, through oracle/_ref's
                   harness; cells of 5 doubles)
  <case>/U         the reference's stored final state, unchanged (2-D: 4 columns, rho w dropped)
  <case>/step      its step count
  <case>/U_here    the final state of the reference compiled here (oracle/_ref/fenice, run as regression.py runs it)
  <case>/ref_diff  how far U_here is from the stored state, in regression.py's measure

The fixtures are test data: nothing of the product reads them.
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

# the regression cases that pin the uniform-mesh path (the reference's names)
CASES = ["isentropic_vortex", "vortex_weno3_rk3", "vortex_weno5_rk3", "hancock_sod", "hancock_taylor_green", "hancock_tgv3d",
         "tgv3d_16", "tgv3d_weno3_rk3", "tgv3d_weno5_rk3", "supersonic_ibm_ghost", "hancock_cylinder", "riemann2d_c3_32",
         "riemann2d_c6_32", "shu_osher", "blast_waves_100", "sod_muscl_vl_rk2", "sod_muscl_mc_rk3_lm", "sod_stiffened_grav",
         "mms_unsteady_hancock", "taylor_green_visc", "cylinder_ibm_ghost", "sphere3d_ibm_ghost", "hancock_sphere3d",
         "cavity_rk3_visc", "cavity_periodic_x", "poiseuille_euler", "sod_1st_euler", "cavity3d_noslip_z", "sod3d_walls_z",
         "sod3d_walls_z_b2", "cavity3d_noslip_z_b2", "cavity_weno3_b2", "cavity_weno5_b2", "cavity3d_weno5_b2", "mms_walls_b2",
         "noh_40", "kelvin_helmholtz_32", "vortex_nrbc", "tgv3d_nrbc"]


def main(ref_root):
    fenice = os.path.join(ROOT, "oracle", "_ref", "fenice")
    os.environ["FENICE_EXE"] = fenice
    sys.path.insert(0, os.path.join(ref_root, "python"))
    sys.path.insert(0, os.path.join(ref_root, "cpp", "tests"))
    import regression  # the reference's table of cases and its runner

    from oracle.oracle import Reference

    tmp = tempfile.mkdtemp(prefix="fvg_regression_")
    out = {}
    for name in CASES:
        tc, ov = regression.CASES[name]
        if tc.startswith("riemann2d:"):
            tc = regression.riemann_case_file(int(tc.split(":")[1]), tmp)
        sets = {} if "boundary_order" in ov else {"boundary_order": 1}   # as regression.run_cpp
        sets.update({k: str(v).replace("{REF}", regression.REF) for k, v in ov.items()})
        cmd = [fenice, "--case", tc, "--no-logo", "--print-config"]
        for k, v in sets.items():
            cmd += ["--set", f"{k}={v}"]
        text = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
        params = {}
        for line in text.splitlines():
            if " = " in line:
                k, v = line.split(" = ", 1)
                params[k.strip()] = v.strip()
        ref = Reference(dict(sets, case=tc))
        U0 = ref.state()
        stored = np.load(os.path.join(regression.REF, f"{name}.npz"))
        U, meta, steps, _ = regression.run_cpp(name, tmp)
        ok, diff, ref_steps = regression.compare(name, U, meta, steps, 1e-8)
        out[f"{name}/params"] = np.array(json.dumps(params))
        out[f"{name}/U0"] = U0
        out[f"{name}/U"] = stored["U"]
        out[f"{name}/step"] = np.array(int(stored["step"]))
        out[f"{name}/U_here"] = U
        out[f"{name}/ref_diff"] = np.array(diff)
        print(f"{name}: {U0.shape[0]} cells, {int(stored['step'])} steps; reference built here vs stored: {diff:.3g} "
              f"({'match' if ok else 'MISMATCH'})")
    np.savez_compressed(os.path.join(HERE, "regression.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FENICE_REFERENCE", "/root/reference"))
