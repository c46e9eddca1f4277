"""The reference's own regression fixtures (its cpp/tests/reference/*.npz final states, extracted with their inputs into
tests/golden/regression.npz by tests/golden/make_regression.py) against the C restatement (oracle/): the same step count
and the reference's own bar (relative difference per variable below 1e-8, cpp/tests/regression.py); and every case's
configuration accepted by the parameter layer."""
import numpy as np
import pytest

import regression_cases as rc
from fenice_b200 import params as fparams
from oracle.oracle import Oracle, not_covered, resolved

FX = rc.load()
NAMES = rc.names(FX)


def test_fixture_bundle():
    assert len(NAMES) == 39
    for n in NAMES:
        assert FX[f"{n}/U0"].shape[1] == 5
        assert FX[f"{n}/U"].shape[0] == FX[f"{n}/U0"].shape[0]
        # the reference compiled from its sources reproduces its stored states within its own bar
        assert float(FX[f"{n}/ref_diff"]) < rc.TOL, n


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_reference_regression_state(name):
    p = rc.params(FX, name)
    why = not_covered(resolved(p))
    if why:
        pytest.skip(f"the restatement does not cover {why} (pinned by the GPU path against the reference instead)")
    try:
        U, t, dts, _, _ = Oracle().run(p, FX[f"{name}/U0"], 1_000_000, 0.0, float(p["t_end"]))
    except ValueError as e:   # e.g. the 2-D viscous sweep, the mass-flow inlet, the non-reflecting outlet
        pytest.skip(f"{e} (pinned by the GPU path against the reference instead)")
    assert len(dts) == int(FX[f"{name}/step"])
    d = rc.rel_diff(U, FX[f"{name}/U"])
    assert d < rc.TOL, d
    # and the restatement equals the reference compiled here
    assert rc.bits_equal(U[:, : FX[f"{name}/U_here"].shape[1]], FX[f"{name}/U_here"])


def test_parameter_layer_accepts_every_case():
    for n in NAMES:   # (the case-file source terms included: they run on the device)
        assert fparams.not_on_device(rc.params(FX, n)) is None, n
        fparams.to_config(rc.params(FX, n))
