"""Host side of the case-file source terms and time-dependent boundary values: the configuration the library gets
(fvg_config's source / boundary_* / param_* fields), the reader of boundary time tables (read_time_table,
cpp/src/SimulationInternal.hpp:62-99), and the library's refusals, checked without a GPU where they come before any
device call."""
import ctypes
import json
import os

import numpy as np
import pytest

from fenice_b200 import params as P
from fenice_b200 import runtime

FX = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sources.npz"))
NAMES = sorted({k.split("/")[0] for k in FX.files if k.endswith("/params")})


def params_of(name, tmp_path):
    p = json.loads(str(FX[f"{name}/params"]))
    for k, v in list(p.items()):
        if k.endswith("_table"):
            (tmp_path / v).write_text(str(FX[f"table/{v}"]))
            p[k] = str(tmp_path / v)
    return p


@pytest.mark.parametrize("name", NAMES)
def test_configuration_carries_the_expressions(name, tmp_path):
    p = params_of(name, tmp_path)
    c = P.to_config(p)
    for q, key in enumerate(P.SOURCE_KEYS):
        assert c.source[q].decode() == str(p.get(key, "0"))
    for k, key in enumerate(P.BOUNDARY_KEYS):
        table = p.get(key + "_table")
        if table:
            rows = P.read_time_table(table)
            assert c.boundary_table_rows[k] == len(rows)
            assert [c.boundary_table[k][i] for i in range(2 * len(rows))] == [x for r in rows for x in r]
        elif P._num(p.get(key, 0.0)) is None:
            assert c.boundary_expr[k].decode() == p[key]
    names = {c.param_names[i].decode(): c.param_values[i] for i in range(c.nparams)}
    assert names["gamma"] == 1.4 and "x" not in names and "t" not in names


def test_time_table_reader(tmp_path):
    f = tmp_path / "t.csv"
    f.write_bytes(b"\xef\xbb\xbf# comment\n\nTime,Value\n0, 1\n0.5 2\n1.0,\t4\n")
    assert P.read_time_table(str(f)) == [(0.0, 1.0), (0.5, 2.0), (1.0, 4.0)]
    for bad, msg in (("0,1\n", "at least two"), ("0,1\n0,2\n", "strictly increasing"), ("0,1\n1,2,3\n", "more than two"),
                     ("0,1\n1,inf\n", "finite"), ("0,1\nx,2\n", "must contain t,value")):
        f.write_text(bad)
        with pytest.raises(ValueError, match=msg):
            P.read_time_table(str(f))


def test_table_and_expression_of_one_value_are_refused(tmp_path):
    f = tmp_path / "u.csv"
    f.write_text("0,1\n1,2\n")
    with pytest.raises(ValueError, match="cannot both be set"):
        P.to_config({"u_in": "1 + t", "u_in_table": str(f)})


def test_reynolds_sets_mu_from_the_inflow_at_t0(tmp_path):
    f = tmp_path / "u.csv"
    f.write_text("0,2.0\n1,3.0\n")
    c = P.to_config({"reynolds": 100.0, "ibm_radius": 0.25, "rho_in": "1.5 + t", "u_in_table": str(f)})
    assert c.mu == 1.5 * 2.0 * 0.5 / 100.0
    with pytest.raises(ValueError, match="reynolds needs positive"):
        P.to_config({"reynolds": 100.0, "u_in": 0.0})


def _create_error(params, **kw):
    lib = runtime.load_library()
    c = P.to_config(params, **kw)
    h = ctypes.c_void_p()
    rc = lib.fvg_create(ctypes.byref(c), ctypes.byref(h))
    return rc, lib.fvg_create_error().decode()


@pytest.mark.parametrize("params, msg", [
    ({"nx": 8, "ny": 8, "source_E": "x +"}, "source_E: cannot evaluate"),
    ({"nx": 8, "ny": 8, "source_mz": "0.1*x"}, "source_mz must be 0 on a 2-D mesh"),
    ({"nx": 8, "ny": 8, "p_out": "t - 1"}, "must be positive at t=0"),
    ({"nx": 8, "ny": 8, "u_in": "1/0*t"}, "non-finite"),
    ({"nx": 8, "ny": 8, "rho_in": 0.0}, "rho_in and p_out must be positive"),
])
def test_library_refuses_before_the_device(params, msg):
    rc, err = _create_error(params)
    assert rc == runtime.FVG_ERR_CONFIG and msg in err, (rc, err)


def test_mixed_precision_refuses_expressions():
    rc, err = _create_error({"nx": 8, "ny": 8, "reconstruction": "muscl", "time_scheme": "rk2", "source_rho": "0.1"}, precision=1)
    assert rc == runtime.FVG_ERR_CONFIG and "FP64 form only" in err
