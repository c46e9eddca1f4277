"""The reference's regression fixtures (tests/golden/regression.npz, made by tests/golden/make_regression.py from the
reference's cpp/tests/reference/*.npz) and the measure its cpp/tests/regression.py compares states with."""
import json
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "regression.npz")
TOL = 1e-8   # cpp/tests/regression.py: --tol default

# cases whose configuration switches on a reference feature the device path refuses (with the refusal's subject): none
NOT_ON_DEVICE = {}
# cases whose source terms read t, evaluated on the device at every stage time with CUDA's transcendental functions
# (each within its documented ulp bound of the C library's the reference calls): their states match the reference's
# within DEVICE_MATH_TOL instead of bit for bit
DEVICE_MATH = {"mms_unsteady_hancock"}
DEVICE_MATH_TOL = 1e-12


def load():
    return np.load(PATH)


def names(fx=None):
    fx = load() if fx is None else fx
    return [k[: -len("/params")] for k in fx.files if k.endswith("/params")]


def params(fx, name):
    return json.loads(str(fx[f"{name}/params"]))


def rel_diff(U, ref):
    """max over cells and variables of |U - ref| / max|ref| of the variable (regression.py's compare); U may carry the
    5th (rho w) column of a 2-D state, which the stored 2-D states drop."""
    ref = np.asarray(ref)
    U = np.asarray(U)[:, : ref.shape[1]]
    scale = np.maximum(np.max(np.abs(ref), axis=0), 1e-30)
    return float(np.max(np.abs(U - ref) / scale))


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
