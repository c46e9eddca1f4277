"""The reference's full Mach 2 cylinder run (1600 x 2400, MUSCL-Hancock with the immersed body, 20 000 steps): its final
time, bow-shock stand-off, loads and the SHA-256 of its final state, written to tests/golden/c5_full.json.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_c5_full.py

Runs the reference compiled from its sources (oracle/_ref, through oracle/ref/ref_harness.cpp) on the host cores; about
50 minutes on 8 cores. The fixture is test data: nothing of the product reads it.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fenice_b200 import diagnostics as D  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

NX, NY, STEPS = 1600, 2400, 20000


def main():
    q = D.cylinder_params(NX, NY, "plain")
    ref = Reference(q, initial_state=(D.RHO_IN, q["u_in"], 0.0, D.P_IN))
    t0 = time.time()
    done = 0
    while done < STEPS:
        done += len(ref.steps(min(1000, STEPS - done), 1e30)[0])
        print(done, ref.t, round(time.time() - t0, 1), flush=True)
    U = ref.state()
    f = ref.ibm_loads()
    qA = 0.5 * D.RHO_IN * q["u_in"] ** 2
    out = {"nx": NX, "ny": NY, "steps": done, "t": ref.t, "wall_s": round(time.time() - t0, 1), "threads": len(os.sched_getaffinity(0)),
           "standoff_over_diameter": D.bow_shock_standoff(U, q), "Fx": f[0], "Fy": f[1], "Mz": f[2], "Cd": f[0] / qA,
           "state_sha256": hashlib.sha256(np.ascontiguousarray(U).tobytes()).hexdigest()}
    with open(os.path.join(HERE, "c5_full.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(out)


if __name__ == "__main__":
    main()
