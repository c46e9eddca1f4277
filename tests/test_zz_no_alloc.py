"""fvg_residual_noalloc, the residual entry point that allocates no device memory (for callers that must not call
cudaMalloc, e.g. inside a framework that owns all device allocations), against the regular entry point fvg_residual.

Through the C ABI: the caller's device buffers are a run's state planes (fvg_device_state) and an output array this test
allocates; two calls in a row on different states must each give fvg_residual's residual and wave speed bit for bit (the
tolerance of every parity test here). The file is collected last so that a failure here leaves every other test run."""
import ctypes
import json

import numpy as np
import pytest

import cases
from fenice_b200 import Run
from fenice_b200 import params as P
from fenice_b200 import runtime as RT

pytestmark = pytest.mark.gpu


def noalloc(params, U_ptr, plane, R_ptr):
    lib = RT.load_library()
    cfg = P.to_config(params)
    s = ctypes.c_double(-1.0)
    rc = lib.fvg_residual_noalloc(ctypes.byref(cfg), ctypes.c_void_p(U_ptr), plane, ctypes.c_void_p(R_ptr), ctypes.byref(s), None)
    return rc, s.value, lib.fvg_create_error().decode()


def planes_to_cells(R_dev, nvar, plane, ncells):
    R = R_dev.cpu().numpy().reshape(nvar, plane)[:, :ncells].T
    out = np.zeros((ncells, 5))
    out[:, :nvar] = R
    return out


@pytest.mark.parametrize("name", ["weno5_hllc_mixed", "w5_3d_periodic_lowmach", "muscl_mc_inlet"])
def test_noalloc_matches_fvg_residual_twice(golden, name):
    import torch

    g = golden[0]
    params = json.loads(str(g[f"{name}/params"]))
    if str(params.get("time_scheme", "auto")).lower() == "auto" and int(params.get("nz", 1)) > 1:
        params["time_scheme"] = "SSP Runge-Kutta 3"
    seed = [c[2] for c in cases.RESIDUAL_CASES if c[0] == name][0]
    states = [g[f"{name}/U"], cases.case_field(params, seed + 1000)]
    run = Run(params)
    ptr, plane, nvar = run.device_state()
    R_dev = torch.empty(nvar * plane, dtype=torch.float64, device="cuda")
    for U in states:   # two calls in a row; the second finds the scratch array as the first left it
        run.set_state(U)
        R_ref, s_ref = run.residual()
        R_dev.fill_(float("nan"))
        torch.cuda.synchronize()
        rc, s, msg = noalloc(params, ptr, plane, R_dev.data_ptr())
        assert rc == RT.FVG_OK, msg
        R = planes_to_cells(R_dev, nvar, plane, run.ncells)
        assert np.array_equal(R.view(np.uint64), R_ref.view(np.uint64)), np.nanmax(np.abs(R - R_ref))
        assert s == s_ref


def test_noalloc_rejects_what_it_cannot_hold():
    import torch

    U = torch.zeros(8, dtype=torch.float64, device="cuda")
    big = dict(nx=330, ny=330, nz=330, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3")   # 68921 tiles > 65536
    rc, _, msg = noalloc(big, U.data_ptr(), 330 ** 3, U.data_ptr())
    assert rc == RT.FVG_ERR_CONFIG and "65536" in msg
    visc = dict(nx=16, ny=16, nz=16, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", use_viscous=True)
    rc, _, msg = noalloc(visc, U.data_ptr(), 16 ** 3, U.data_ptr())
    assert rc == RT.FVG_ERR_CONFIG and "viscous" in msg
