"""Initial conditions from case files (fenice_b200.casefile) against the reference's own evaluation of the same case
files (tests/golden/initial.npz, written by tests/golden/make_initial.py): bit for bit, transcendental functions
included (the library's expression compiler calls the C library's functions, as the reference's TinyExpr does); the
expression grammar's refusals."""
import json
import os
import tempfile

import numpy as np
import pytest

from fenice_b200 import casefile

FX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "initial.npz"))
NAMES = [k[: -len("/case_toml")] for k in FX.files if k.endswith("/case_toml")]


def load(name):
    tmp = tempfile.mkdtemp(prefix="fvg_case_")
    path = os.path.join(tmp, "case.toml")
    with open(path, "w") as f:
        f.write(str(FX[f"{name}/case_toml"]))
    return casefile.load(path, json.loads(str(FX[f"{name}/overrides"])))


@pytest.mark.parametrize("name", NAMES)
def test_initial_state_matches_the_reference(name):
    params, U = load(name)
    ref = FX[f"{name}/U0"]
    assert U.shape == ref.shape
    assert np.array_equal(U.view(np.uint64), ref.view(np.uint64)), np.abs(U - ref).max()


def test_expression_grammar():
    names = [("Lx", 3.0)]
    ev = lambda src: casefile.Expr(src, names, "t")(0.5, 0.0, 0.0)[0]   # noqa: E731
    assert ev("2^3^2") == 2.0 ** 9            # right-associative power
    assert ev("-2^2") == -4.0
    assert ev("log(1000)") == 3.0              # base 10, ln is natural
    assert abs(ev("ln(e)") - 1.0) < 1e-15
    assert ev("Lx/2 + x") == 2.0
    assert casefile.Expr("0.3", names, "t")(0.0, 0.0, 0.0) == 0.3
    for bad in ("__import__('os')", "x.real", "[1, 2]", "foo(1)", "q + 1", "lambda: 1"):
        with pytest.raises(ValueError):
            casefile.Expr(bad, names, "t")


def test_profiles_are_refused():
    with pytest.raises(ValueError, match="profile"):
        casefile.initial_state({"profile": "isentropic_vortex"}, dict(nx=4, ny=4))


def test_a_3d_case_needs_a_3d_mesh():
    with pytest.raises(ValueError, match="3-D"):
        casefile.initial_state({"state": {"rho": 1.0, "p": 1.0}}, dict(nx=4, ny=4), three_d_case=True)


def test_a_2d_case_on_a_3d_mesh_is_one_layer_extruded():
    U = casefile.initial_state({"state": {"rho": "1 + x + y + z", "p": 1.0}}, dict(nx=4, ny=3, nz=5, Lz=2.0))
    layers = U.reshape(5, 12, 5)
    assert all(np.array_equal(layers[0], layers[k]) for k in range(5))
    assert np.array_equal(U[:12, 0], casefile.initial_state({"state": {"rho": "1 + x + y", "p": 1.0}}, dict(nx=4, ny=3))[:, 0])
