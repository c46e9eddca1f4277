"""The reference's own regression fixtures (its cpp/tests/reference/*.npz, with their inputs, in
tests/golden/regression.npz) run through the device path: every case the device computes reaches the reference's step
count and its final state within the reference's bar (relative difference per variable below 1e-8,
cpp/tests/regression.py), and equals bit for bit the reference compiled from its sources (the fixture's U_here), except
a case whose source terms read t: evaluated on the device with CUDA's functions at every stage, its state is within
1e-12 (relative, per variable) of the reference's."""
import numpy as np
import pytest

import regression_cases as rc
from fenice_b200 import Run

pytestmark = pytest.mark.gpu

FX = rc.load()
NAMES = rc.names(FX)


@pytest.mark.parametrize("name", [n for n in NAMES if n not in rc.NOT_ON_DEVICE])
def test_device_reproduces_reference_regression_state(name):
    p = rc.params(FX, name)
    run = Run(p, U=FX[f"{name}/U0"])
    steps = run.run(float(p["t_end"]), max_steps=int(p.get("max_steps", 0) or 0))
    assert steps == int(FX[f"{name}/step"])
    U = run.state()
    d = rc.rel_diff(U, FX[f"{name}/U"])
    here = FX[f"{name}/U_here"]
    exact = rc.bits_equal(U[:, : here.shape[1]], here)
    d_here = rc.rel_diff(U, here)
    print(f"\n{name}: {steps} steps, relative difference from the stored state {d:.3g}, "
          f"bit-exact vs the reference compiled here: {exact} (relative difference {d_here:.3g})")
    assert d < rc.TOL
    if name in rc.DEVICE_MATH:
        assert d_here < rc.DEVICE_MATH_TOL
    else:
        assert exact
