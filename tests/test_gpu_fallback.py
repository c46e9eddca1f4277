"""positivity_fallback on the GPU against the reference, bit for bit (fixtures tests/golden/fallback.npz): a double
rarefaction and a 3-D blast that the reference only survives with the guard (a stage whose result has a cell without
density or pressure is repeated with first-order faces around the flagged cells), and two problems without repairs (the
guarded run has the unguarded bits); steps one at a time (dt, wave speed) and through the graph-captured loop; and the
unguarded device run diverges where the reference's does."""
import json
import os

import numpy as np
import pytest

import cases
from fenice_b200 import Run

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fallback.npz"))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def describe(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return f"max |diff| {d.max():.3e}, {int((d > 0).sum())} values differ"


@pytest.mark.parametrize("case", cases.FALLBACK_CASES, ids=[c[0] for c in cases.FALLBACK_CASES])
def test_guarded_steps_bit_exact(fx, case):
    name, n = case[0], case[3]
    run = Run(json.loads(str(fx[f"{name}/params"])), U=fx[f"{name}/U0"])
    dts, sms = [], []
    for _ in range(n):
        r = run.step(1e30)
        dts.append(r.dt)
        sms.append(r.s_max)
    assert bits_equal(dts, fx[f"{name}/dts"]), (dts, fx[f"{name}/dts"])
    assert bits_equal(sms, fx[f"{name}/smaxs"])
    assert bits_equal(run.state(), fx[f"{name}/U"]), describe(run.state(), fx[f"{name}/U"])
    assert run.t == float(fx[f"{name}/t"])


@pytest.mark.parametrize("case", cases.FALLBACK_CASES, ids=[c[0] for c in cases.FALLBACK_CASES])
def test_guarded_graph_run_and_unguarded_run(fx, case):
    name, n = case[0], case[3]
    params = json.loads(str(fx[f"{name}/params"]))
    run = Run(params, U=fx[f"{name}/U0"])
    assert run.run(1e30, max_steps=n) == n
    assert bits_equal(run.state(), fx[f"{name}/U"]), describe(run.state(), fx[f"{name}/U"])
    plain = Run(dict(params, positivity_fallback=False), U=fx[f"{name}/U0"])
    if str(fx[f"{name}/unguarded"]) == "diverges":
        with pytest.raises(RuntimeError, match="diverged"):
            plain.run(1e30, max_steps=n)
    else:
        assert plain.run(1e30, max_steps=n) == n
        assert bits_equal(plain.state(), fx[f"{name}/U"])
