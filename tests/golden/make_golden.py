"""Writes the golden fixtures of the parity tests with the reference solver itself.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_golden.py

Runs the reference compiled from its own sources (oracle/_ref/libfenice_ref.so, through oracle/ref/ref_harness.cpp) on
the seeded inputs of tests/cases.py and stores, per case, the parameters, the input state and the reference's output:
  residuals.npz  one residual R(U) and its wave speed (Simulation::residual, with the MUSCL-Hancock predictor where the
                 case has a half step)
  steps.npz      the state after n steps of the serial time loop, with each step's dt and wave speed
  ibm.npz        immersed-body cases: the forced field, a residual, then a few steps
  visc2d.npz     2-D viscous cases (NavierStokes::viscous_residual_rows): a residual, then a few steps
  hancock3d.npz  3-D MUSCL-Hancock (MusclReconstruction::hancock_residual_3d): residuals with the predictor, then steps
  forces.npz     the body force (ConstantBodyForce) and MUSCL-Hancock with viscous fluxes: a residual, then steps
  fallback.npz   positivity_fallback: steps of problems that need repairs (and of two that need none), with and without the
                 guard (the unguarded reference diverges on the first two)
  riemann.json   the reference's bench_riemann fingerprints over one pass of its 65536 state pairs
                 (oracle/_ref/bench_riemann 65536)
Sections can be named on the command line (residuals steps ibm visc2d hancock3d forces fallback riemann); default: all.
The fixtures are test data: nothing of the product reads them.
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.oracle import Reference  # noqa: E402
import cases  # noqa: E402


def visc2d():
    out = {}
    for name, params, seed, n in cases.VISC2D_CASES:
        U = cases.case_field(params, seed)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        R, s = ref.residual(U)
        out[f"{name}/params"] = np.array(json.dumps(params))
        out[f"{name}/U0"] = U
        out[f"{name}/R"] = R
        out[f"{name}/smax"] = np.array(s)
        ref.set_state(U)
        dts, sms = ref.steps(n, 1e30)
        out[f"{name}/U"] = ref.state()
        out[f"{name}/dts"] = dts
        out[f"{name}/smaxs"] = sms
        out[f"{name}/t"] = np.array(ref.t)
        print(f"visc2d {name}: smax {s:.6g}, {len(dts)} steps")
    np.savez_compressed(os.path.join(HERE, "visc2d.npz"), **out)


def hancock3d():
    out = {}
    for name, params, seed, half in cases.HANCOCK3D_RESIDUAL_CASES:
        U = cases.case_field(params, seed)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        R, s = ref.residual(U, predictor_half_dt=half)
        out[f"{name}/params"] = np.array(json.dumps(params))
        out[f"{name}/U"] = U
        out[f"{name}/R"] = R
        out[f"{name}/smax"] = np.array(s)
        out[f"{name}/half_dt"] = np.array(half)
        print(f"hancock3d residual {name}: smax {s:.6g}")
    for name, params, seed, n in cases.HANCOCK3D_STEP_CASES:
        U = cases.case_field(params, seed)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        ref.set_state(U)
        dts, sms = ref.steps(n, 1e30)
        out[f"{name}/params"] = np.array(json.dumps(params))
        out[f"{name}/U0"] = U
        out[f"{name}/U"] = ref.state()
        out[f"{name}/dts"] = dts
        out[f"{name}/smaxs"] = sms
        out[f"{name}/t"] = np.array(ref.t)
        print(f"hancock3d steps {name}: {len(dts)} steps, t = {ref.t:.6g}")
    np.savez_compressed(os.path.join(HERE, "hancock3d.npz"), **out)


def forces():
    out = {}
    for name, params, seed, half, n in cases.FORCE_CASES:
        U = cases.case_field(params, seed)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        R, s = ref.residual(U, predictor_half_dt=half)
        out[f"{name}/params"] = np.array(json.dumps(params))
        out[f"{name}/U0"] = U
        out[f"{name}/R"] = R
        out[f"{name}/smax"] = np.array(s)
        out[f"{name}/half_dt"] = np.array(half)
        ref.set_state(U)
        dts, sms = ref.steps(n, 1e30)
        out[f"{name}/U"] = ref.state()
        out[f"{name}/dts"] = dts
        out[f"{name}/smaxs"] = sms
        out[f"{name}/t"] = np.array(ref.t)
        print(f"forces {name}: smax {s:.6g}, {len(dts)} steps")
    np.savez_compressed(os.path.join(HERE, "forces.npz"), **out)


def fallback():
    out = {}
    for name, params, spec, n in cases.FALLBACK_CASES:
        U = cases.fallback_state(spec)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        ref.set_state(U)
        dts, sms = ref.steps(n, 1e30)
        out[f"{name}/params"] = np.array(json.dumps(params))
        out[f"{name}/U0"] = U
        out[f"{name}/U"] = ref.state()
        out[f"{name}/dts"] = dts
        out[f"{name}/smaxs"] = sms
        out[f"{name}/t"] = np.array(ref.t)
        plain = Reference(dict(params, positivity_fallback=False), initial_state=(1, 0, 0, 1, 0))
        plain.set_state(U)
        try:
            plain.steps(n, 1e30)
            unguarded = "same" if np.array_equal(plain.state().view(np.uint64), ref.state().view(np.uint64)) else "differs"
        except RuntimeError:
            unguarded = "diverges"
        out[f"{name}/unguarded"] = np.array(unguarded)
        print(f"fallback {name}: {len(dts)} steps, t = {ref.t:.6g}; without the guard the reference {unguarded}")
    np.savez_compressed(os.path.join(HERE, "fallback.npz"), **out)


def main(sections=("residuals", "steps", "ibm", "visc2d", "hancock3d", "forces", "fallback", "riemann")):
    if "visc2d" in sections:
        visc2d()
    if "hancock3d" in sections:
        hancock3d()
    if "forces" in sections:
        forces()
    if "fallback" in sections:
        fallback()
    if "residuals" in sections:
        residuals()
    if "steps" in sections:
        steps()
    if "ibm" in sections:
        ibm()
    if "riemann" in sections:
        riemann()


def residuals():
    res = {}
    for name, params, seed, half in cases.RESIDUAL_CASES:
        U = cases.case_field(params, seed)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        R, s = ref.residual(U, predictor_half_dt=half)
        res[f"{name}/params"] = np.array(json.dumps(params))
        res[f"{name}/U"] = U
        res[f"{name}/R"] = R
        res[f"{name}/smax"] = np.array(s)
        res[f"{name}/half_dt"] = np.array(half)
        print(f"residual {name}: smax {s:.6g}")
    np.savez_compressed(os.path.join(HERE, "residuals.npz"), **res)


def steps():
    st = {}
    for name, params, seed, n in cases.STEP_CASES:
        U = cases.case_field(params, seed)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        ref.set_state(U)
        dts, sms = ref.steps(n, 1e30)
        st[f"{name}/params"] = np.array(json.dumps(params))
        st[f"{name}/U0"] = U
        st[f"{name}/U"] = ref.state()
        st[f"{name}/dts"] = dts
        st[f"{name}/smaxs"] = sms
        st[f"{name}/t"] = np.array(ref.t)
        print(f"steps {name}: {len(dts)} steps, t = {ref.t:.6g}")
    np.savez_compressed(os.path.join(HERE, "steps.npz"), **st)


def ibm():
    ib = {}
    for name, params, W0, seed, n in cases.IBM_CASES:
        ref = Reference(params, initial_state=W0)
        U = cases.ibm_field(params, W0, seed)
        ref.set_state(U, force_ibm=True)   # the body forced as initialize_field forces it
        U = ref.state()
        half = 0.002 if str(params.get("time_scheme")) == "MUSCL-Hancock" else 0.0
        R, s = ref.residual(U, predictor_half_dt=half)
        ib[f"{name}/params"] = np.array(json.dumps(params))
        ib[f"{name}/U0"] = U
        ib[f"{name}/R"] = R
        ib[f"{name}/smax"] = np.array(s)
        ib[f"{name}/half_dt"] = np.array(half)
        ib[f"{name}/mask"] = ref.solid_mask()
        dts, sms = ref.steps(n, 1e30)
        ib[f"{name}/U"] = ref.state()
        ib[f"{name}/dts"] = dts
        ib[f"{name}/smaxs"] = sms
        ib[f"{name}/t"] = np.array(ref.t)
        print(f"ibm {name}: {int(ib[f'{name}/mask'].sum())} solid cells, {len(dts)} steps")
    np.savez_compressed(os.path.join(HERE, "ibm.npz"), **ib)


def riemann():
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "bench_riemann"), "65536"], capture_output=True, text=True, check=True).stdout
    hashes = {}
    for line in out.splitlines():
        parts = line.split()
        eos, solver = parts[0], " ".join(parts[1:parts.index("ns/call") - 1])
        hashes[f"{eos} {solver}"] = parts[parts.index("hash") + 1]
    with open(os.path.join(HERE, "riemann.json"), "w") as f:
        json.dump({"command": "oracle/_ref/bench_riemann 65536", "hashes": hashes}, f, indent=1)
    print(hashes)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("residuals", "steps", "ibm", "visc2d", "hancock3d", "forces", "fallback", "riemann"))
