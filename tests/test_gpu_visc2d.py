"""The 2-D viscous sweep on the GPU against the reference, bit for bit (fixtures tests/golden/visc2d.npz, written by the
reference's NavierStokes::viscous_residual_rows through tests/golden/make_golden.py): residual and wave speed of a seeded
field, then a few steps, for periodic, no-slip, moving-wall, slip-wall, inlet / outlet and mixed sides, boundary_order 1
and 2, every reconstruction and time scheme; and the mixed-precision form within the L1 bar."""
import json
import os

import numpy as np
import pytest

import cases
from fenice_b200 import Run

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "visc2d.npz"))


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def describe(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return f"max |diff| {d.max():.3e} at {np.unravel_index(d.argmax(), d.shape)}, {int((d > 0).sum())} values differ"


@pytest.mark.parametrize("case", cases.VISC2D_CASES, ids=[c[0] for c in cases.VISC2D_CASES])
def test_visc2d_residual_bit_exact(fx, case):
    name = case[0]
    run = Run(json.loads(str(fx[f"{name}/params"])), U=fx[f"{name}/U0"])
    R, s = run.residual()
    assert bits_equal(R, fx[f"{name}/R"]), describe(R, fx[f"{name}/R"])
    assert s == float(fx[f"{name}/smax"])


@pytest.mark.parametrize("case", cases.VISC2D_CASES, ids=[c[0] for c in cases.VISC2D_CASES])
def test_visc2d_steps_bit_exact(fx, case):
    name, _, _, n = case
    run = Run(json.loads(str(fx[f"{name}/params"])), U=fx[f"{name}/U0"])
    assert run.run(1e30, max_steps=n) == n
    assert bits_equal(run.state(), fx[f"{name}/U"]), describe(run.state(), fx[f"{name}/U"])
    assert run.t == float(fx[f"{name}/t"])


def test_visc2d_mixed_form(fx):
    name = "v2_periodic_weno5_rk3"
    params = json.loads(str(fx[f"{name}/params"]))
    plain = Run(params, U=fx[f"{name}/U0"])
    mixed = Run(params, U=fx[f"{name}/U0"], precision=1)
    plain.run(1e30, max_steps=20)
    mixed.run(1e30, max_steps=20)
    l1 = np.abs(mixed.state()[:, 0] - plain.state()[:, 0]).sum() / np.abs(plain.state()[:, 0]).sum()
    print(f"\n2-D viscous, mixed vs FP64 after 20 steps: L1(rho) {l1:.2e}")
    assert l1 <= 1e-4
