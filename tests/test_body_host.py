"""Immersed bodies in motion: the configurations the library refuses before any device call, with the reference's
parameter checks (cpp/src/Params.cpp:505-546), and the parameter layer's reading of the motion keys."""
import ctypes

import pytest

from fenice_b200 import params as P
from fenice_b200 import runtime

BASE = dict(nx=16, ny=16, reconstruction="muscl", time_scheme="SSP Runge-Kutta 2", use_ibm=True, ibm_shape="Cylinder", ibm_radius=0.2)


def create(params):
    lib = runtime.load_library()
    c = P.to_config(params)
    h = ctypes.c_void_p()
    rc = lib.fvg_create(ctypes.byref(c), ctypes.byref(h))
    return rc, lib.fvg_create_error().decode()


def test_motion_keys_reach_the_configuration():
    c = P.to_config(dict(BASE, ibm_vx=0.5, ibm_mass=2.0, ibm_damp_x=0.1, ibm_inertia=1.0, ibm_cm_x=0.1, ibm_cm_y=0.0))
    assert (c.ibm_vx, c.ibm_mass, c.ibm_damp_x, c.ibm_inertia, c.ibm_cm_given, c.ibm_cm_x) == (0.5, 2.0, 0.1, 1.0, 1, 0.1)
    assert P.to_config(dict(BASE, use_ibm=False, ibm_vx=0.5)).ibm_vx == 0.0   # (no body, no motion)
    with pytest.raises(ValueError, match="go together"):
        P.to_config(dict(BASE, ibm_cm_x=0.1))


@pytest.mark.parametrize("over, msg", [
    (dict(ibm_stiff_x=1.0), "set ibm_mass > 0"),
    (dict(ibm_damp_theta=1.0), "set ibm_inertia > 0"),
    (dict(ibm_mass=1.0, ibm_cm_x=0.1, ibm_cm_y=0.0), "both driven"),
    (dict(ibm_mass=1.0, ibm_inertia=0.001, ibm_cm_x=0.1, ibm_cm_y=0.0), "must exceed ibm_mass"),
    (dict(ibm_mass=1.0, ibm_omega=1.0), "translates only"),
    (dict(ibm_inertia=1.0, ibm_vx=1.0), "pinned at its placement"),
    (dict(ibm_inertia=1.0, ibm_omega=1.0, ibm_omega_from=0.1), "prescribed rotation"),
    (dict(ibm_mass=1.0, time_scheme="MUSCL-Hancock"), "Runge-Kutta or Euler"),
    (dict(ibm_omega_from=0.1), "need a rotation"),
    (dict(ibm_omega=1.0, ibm_omega_from=0.2, ibm_omega_until=0.1), "later than"),
    (dict(nz=8, ibm_vx=1.0, ibm_shape="Cylinder"), "a sphere"),
    (dict(ibm_omega_x=1.0), "3-D mesh"),
    (dict(ibm_vz=1.0, ibm_vx=1.0), "ibm_vz needs a 3-D mesh"),
])
def test_refusals(over, msg):
    rc, err = create(dict(BASE, **over))
    assert rc == runtime.FVG_ERR_CONFIG and msg in err, (rc, err)
