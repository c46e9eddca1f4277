"""The case-file expression compiler (fenice_b200/csrc/expr.cu) against the reference's own expression engine
(tests/golden/expr.json, written by tests/golden/make_expr.py from the reference's TinyExpr): the same expressions
accepted and refused, and on the host the same values bit for bit, transcendental functions included (both call the C
library)."""
import json
import os
import struct

import numpy as np
import pytest

from fenice_b200 import runtime

FX = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "expr.json")))
POINTS = np.array([[struct.unpack("<d", bytes.fromhex(h))[0] for h in p] for p in FX["points"]])


def bits(hexes):
    return np.array([struct.unpack("<d", bytes.fromhex(h))[0] for h in hexes]).view(np.uint64)


@pytest.mark.parametrize("case", FX["cases"], ids=[c["expr"] or "<empty>" for c in FX["cases"]])
def test_expression_matches_the_reference(case):
    names = dict(FX["names"])
    if case["refused"]:
        with pytest.raises(ValueError, match="cannot evaluate"):
            runtime.eval_expression(case["expr"], names, POINTS[:, 0], POINTS[:, 1], POINTS[:, 2], 0.0)
        return
    got = np.array([runtime.eval_expression(case["expr"], names, [x], [y], [z], t)[0] for x, y, z, t in POINTS])
    want = bits(case["values"])
    same = (got.view(np.uint64) == want) | (np.isnan(got) & np.isnan(want.view(np.float64)))
    assert same.all(), (case["expr"], got, want.view(np.float64))


def test_later_names_replace_earlier_ones():
    assert runtime.eval_expression("a*2", [("a", 1.0), ("a", 3.0)], [0.0], [0.0], [0.0], 0.0)[0] == 6.0


def test_whole_numbers_are_exact():
    # a whole number is read with strtod (correctly rounded); inside an expression the engine's own reading applies
    assert runtime.eval_expression("0.3", {}, [0.0], [0.0], [0.0], 0.0)[0] == 0.3
    assert runtime.eval_expression("0.3 + 0", {}, [0.0], [0.0], [0.0], 0.0)[0] == 3 * 0.1
