"""flux_quadrature = fourth: the configurations the library refuses before any device call, as the reference's
parameter checks do (cpp/src/Params.cpp:448-467), and the parameter layer's reading of the key."""
import ctypes

import pytest

from fenice_b200 import params as P
from fenice_b200 import runtime

BASE = dict(nx=8, ny=8, reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", flux_quadrature="fourth")


def create(params, part=None, **kw):
    lib = runtime.load_library()
    c = P.to_config(params, **kw)
    h = ctypes.c_void_p()
    rc = lib.fvg_create(ctypes.byref(c), ctypes.byref(h)) if part is None else lib.fvg_create_part(ctypes.byref(c), part[0], part[1], ctypes.byref(h))
    return rc, lib.fvg_create_error().decode()


def test_key_is_read():
    assert P.to_config(BASE).flux_quadrature == 1
    assert P.to_config(dict(BASE, flux_quadrature="midpoint")).flux_quadrature == 0
    with pytest.raises(ValueError, match="midpoint or fourth"):
        P.to_config(dict(BASE, flux_quadrature="gauss"))


@pytest.mark.parametrize("over, msg", [
    (dict(reconstruction="muscl", time_scheme="rk2"), "needs reconstruction = weno3 or weno5"),
    (dict(use_ibm=True), "immersed body"),
    (dict(positivity_fallback=True), "positivity_fallback needs flux_quadrature = midpoint"),
])
def test_refusals(over, msg):
    rc, err = create(dict(BASE, **over))
    assert rc == runtime.FVG_ERR_CONFIG and msg in err, (rc, err)


def test_mixed_precision_and_parts_are_refused():
    rc, err = create(BASE, precision=1)
    assert rc == runtime.FVG_ERR_CONFIG and "FP64 form only" in err
    rc, err = create(dict(BASE, nx=8, ny=16), part=(2, 0))
    assert rc == runtime.FVG_ERR_CONFIG and "serial" in err
