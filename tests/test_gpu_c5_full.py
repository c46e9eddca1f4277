"""The full Mach 2 cylinder (1600 x 2400 cells, MUSCL-Hancock with the immersed body, 20 000 steps, about 20 s on a B200)
against the reference's own run of it: the same final time and the same final state, by SHA-256 of its 3 840 000 x 5
doubles (fixture tests/golden/c5_full.json, written by tests/golden/make_c5_full.py with the reference compiled from its
sources), hence the same bow-shock stand-off and drag."""
import hashlib
import json
import os

import numpy as np
import pytest

from fenice_b200 import Run
from fenice_b200 import diagnostics as D

pytestmark = pytest.mark.gpu


def test_full_cylinder_run_equals_the_reference():
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c5_full.json")) as f:
        ref = json.load(f)
    q = D.cylinder_params(ref["nx"], ref["ny"], "plain")
    run = Run(q, U=D.free_stream(q))
    assert run.run(1e30, max_steps=ref["steps"]) == ref["steps"]
    U = run.state()
    loads = run.ibm_loads()
    print(f"\nC5 full run: t = {run.t}, stand-off / D = {D.bow_shock_standoff(U, q):.6f}, Cd = {loads['Cd']:.6f}")
    assert run.t == ref["t"]
    assert hashlib.sha256(np.ascontiguousarray(U).tobytes()).hexdigest() == ref["state_sha256"]
    assert loads["Cd"] == ref["Cd"]
    run.close()
