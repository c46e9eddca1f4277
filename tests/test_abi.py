"""The C ABI library without a GPU: it loads, exports every entry point include/fenice_gpu.h declares, and rejects the
configurations the reference rejects or the device path does not support before it touches CUDA; the Python host layer
parses the reference's parameter names the way the reference does."""
import ctypes
import os
import re

import pytest

from fenice_b200 import params as P
from fenice_b200 import runtime as RT

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    with open(os.path.join(ROOT, "include", "fenice_gpu.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(fvg_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = RT.load_library()
    names = header_functions()
    assert names, "no entry points parsed from the header"
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(RT.EXPORTS)
    assert lib.fvg_abi_version() == 9


def create_code(params):
    lib = RT.load_library()
    params = dict(params)
    c = P.to_config(params, precision=1 if params.pop("precision_mixed", False) else 0)
    h = ctypes.c_void_p()
    rc = lib.fvg_create(ctypes.byref(c), ctypes.byref(h))
    return rc, lib.fvg_create_error().decode()


@pytest.mark.parametrize("params,words", [
    (dict(nx=0), "nx"),
    (dict(bc_xmin="periodic", bc_xmax="wall"), "periodic"),
    (dict(reconstruction="weno5", time_scheme="MUSCL-Hancock"), "MUSCL-Hancock"),
    (dict(use_bodyforce=True, reconstruction="muscl", time_scheme="SSP Runge-Kutta 2", precision_mixed=True), "FP64 form only"),
    (dict(use_ibm=True, ibm_shape="Cylinder", ibm_radius=0.1, flux_quadrature="fourth", reconstruction="weno5", time_scheme="rk3"), "immersed body"),
    (dict(boundary_order=3), "boundary_order"),
    (dict(cfl=0.0), "cfl"),
])
def test_invalid_configurations_are_rejected_on_the_host(params, words):
    rc, msg = create_code(params)
    assert rc == RT.FVG_ERR_CONFIG
    assert words.lower() in msg.lower()


def test_parameter_names_parse_like_the_reference():
    c = P.to_config({"riemann_solver": "HLLC (Low-Mach Thornber)", "muscl_limiter": "van leer", "reconstruction": "WENO5",
                     "bc_xmin": "Velocity Inlet", "time_scheme": "ssprk3"})
    assert (c.riemann, c.limiter, c.reconstruction, c.bc[0], c.time_scheme) == (1, 1, 3, 3, 2)
    # time_scheme = auto (Params.cpp:360-363)
    assert P.to_config({"reconstruction": "muscl"}).time_scheme == 3
    assert P.to_config({"reconstruction": "muscl", "use_viscous": "true"}).time_scheme == 1
    assert P.to_config({"reconstruction": "weno5"}).time_scheme == 0
    for bad in ({"riemann_solver": "roe"}, {"muscl_limiter": "superbee"}, {"bc_xmin": "slip"}, {"time_scheme": "rk4"}):
        with pytest.raises(ValueError):
            P.to_config(bad)


def test_case_file_keys(tmp_path):
    f = tmp_path / "case.toml"
    f.write_text('[case]\nname = "x"\n[mesh]\nnx = 64\nLx = 2.0\n[numerics]\nreconstruction = "weno5"\ncfl = 0.4\n'
                 '[boundaries]\nbc_xmin = "periodic"\nbc_xmax = "periodic"\n[initial]\nstate = { rho = 1.0, p = 1.0 }\n')
    params, initial = P.load_case(str(f), {"ny": 8})
    assert params == {"nx": 64, "Lx": 2.0, "reconstruction": "weno5", "cfl": 0.4, "bc_xmin": "periodic", "bc_xmax": "periodic", "ny": 8}
    assert initial["state"]["rho"] == 1.0
