"""Values of case-file expressions computed by the reference's own expression engine, for the expression compiler's tests.

    make -C oracle/ref REF=/path/to/fenice -j8 && python tests/golden/make_expr.py

The reference's TinyExpr (built with TE_POW_FROM_RIGHT into oracle/_ref/libfenice_ref.so by oracle/ref/Makefile) is
called through ctypes the way the reference's Evaluator calls it (cpp/src/CaseFile.cpp:299-377): x, y, z, t bound
first, then the named parameters, each a variable; a value that is a whole number for the C library's strtod is that
number (Evaluator::compile), anything else goes through te_compile, then te_eval at every point. An expression that
te_compile refuses is recorded as refused. tests/golden/expr.json holds, per expression, the bound names and values,
the points and the values' bit patterns. The fixtures are test data: nothing of the product reads them.
"""
import ctypes
import json
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libfenice_ref.so")

NAMES = {"Lx": 2.0, "Ly": 1.5, "Lz": 1.0, "nx": 64.0, "ny": 48.0, "nz": 1.0, "gamma": 1.4, "u_in": 0.3, "mu": 0.001, "pr": 0.72,
         "rho_in": 1.2, "p_out": 0.7142857142857143, "a_1": 0.25}

EXPRESSIONS = [
    # numbers as the engine reads them (not always the correctly rounded value of the text)
    "0.3", "0.3*x", "1.1 + x - x", "123.456e-3*x", "1e-300*x", "7e22*x", "0x1F + x", "1e5x" , "3.14159265358979 * x", ".5*x", "5.*x",
    "1e", "x*1e+2", "0.1+0.2+x-x", "2.5e-5*t", "100000000000000000000001*x",
    # precedence and associativity
    "2^3^2", "-2^2", "(-2)^2", "2^-2", "2^-x^2", "-x^2", "-x^-y", "x^y^z", "-x^y^-z", "--x", "-+-x", "2*-x", "x-y-z", "x/y/z",
    "x%0.3", "x - y*z + t/2", "(x+y)*(z-t)", "x^2 + y^2 - 2*x*y",
    # functions, with and without parentheses
    "sin(x)", "sin x", "sin x^2", "sin(x)^2", "sin -x", "sqrt x*y", "cos(2*pi*x/Lx)*sin(2*pi*y/Ly)", "exp(-((x-1)^2 + (y-0.75)^2)/0.01)",
    "atan2(y, x)", "pow(x, y)", "pow(2, 0.5)", "log(x)", "ln(x)", "log10(100*x)", "abs(x - y)", "ceil(x*3)", "floor(-x*3)",
    "tanh(5*(y - Ly/2))", "asin(x/4)", "acos(y/4)", "atan(x)", "cosh(x)", "sinh(y)", "tan(x)", "fac(5)", "fac(x*3)", "ncr(10, 3)",
    "npr(6, 2)", "ncr(x*5, 2)", "e", "e()", "pi", "pi()", "e^x", "2*pi", "exp(1)",
    # logical and comparison operators
    "x > y", "x >= 1", "x < y && y < z", "x == x", "x != y", "!x", "!!x", "-!x", "!-x", "-!!x", "x > 0.5 || y > 0.5", "(x > 1)*2 + 1",
    "1 < 2 == 1", "!0", "!x*3",
    # lists
    "(x, y)", "x, y, z",
    # parameters
    "gamma/(gamma - 1)", "rho_in*u_in*x", "a_1 + Lx*Ly", "mu*sin(t)", "1/(gamma - 1) + 0.5*rho_in*u_in^2",
    # manufactured-solution style sources
    "0.1*pi*cos(pi*(x + y - t))*(1 + 0.2*sin(pi*x))", "-2*mu*pi^2*sin(pi*x)*cos(pi*y)*exp(-2*mu*pi^2*t)",
    # refused
    "x +", "sin", "foo(x)", "x y", "(x", "x)", "atan2(x)", "atan2(x, y, z)", "x = 1", "x & y", "x | y", ".", "", "2**3", "pi(1)",
]


class TeVariable(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("address", ctypes.c_void_p), ("type", ctypes.c_int), ("context", ctypes.c_void_p)]


def hexes(a):
    return [struct.pack("<d", float(v)).hex() for v in a]


def main():
    lib = ctypes.CDLL(LIB)
    lib.te_compile.restype = ctypes.c_void_p
    lib.te_compile.argtypes = [ctypes.c_char_p, ctypes.POINTER(TeVariable), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.te_eval.restype = ctypes.c_double
    lib.te_eval.argtypes = [ctypes.c_void_p]
    lib.te_free.argtypes = [ctypes.c_void_p]
    order = ["x", "y", "z", "t"] + list(NAMES)
    store = (ctypes.c_double * len(order))()
    for i, k in enumerate(order[4:]):
        store[4 + i] = NAMES[k]
    names = [ctypes.c_char_p(k.encode()) for k in order]
    vars_ = (TeVariable * len(order))()
    for i in range(len(order)):
        vars_[i] = TeVariable(names[i].value, ctypes.addressof(store) + 8 * i, 0, None)
    rng = np.random.default_rng(7)
    pts = rng.uniform(0.05, 1.95, size=(12, 4))
    pts[0] = [1.0, 1.0, 0.5, 0.0]
    pts[1] = [0.5, 0.25, 0.125, 1.5]
    libc = ctypes.CDLL(None)
    libc.strtod.restype = ctypes.c_double
    libc.strtod.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
    out = []
    for src in EXPRESSIONS:
        buf = ctypes.create_string_buffer(src.encode())
        end = ctypes.c_char_p()
        number = libc.strtod(buf, ctypes.byref(end))
        if src and ctypes.cast(end, ctypes.c_void_p).value == ctypes.addressof(buf) + len(src.encode()):
            out.append({"expr": src, "refused": False, "values": hexes([number] * len(pts))})
            continue
        err = ctypes.c_int(0)
        e = lib.te_compile(src.encode(), vars_, len(order), ctypes.byref(err))
        if not e:
            out.append({"expr": src, "refused": True})
            continue
        vals = []
        for x, y, z, t in pts:
            store[0], store[1], store[2], store[3] = x, y, z, t
            vals.append(lib.te_eval(e))
        lib.te_free(e)
        out.append({"expr": src, "refused": False, "values": hexes(vals)})
    doc = {"names": NAMES, "points": [hexes(p) for p in pts], "cases": out}
    with open(os.path.join(HERE, "expr.json"), "w") as f:
        json.dump(doc, f, indent=0)
    print(f"{len(out)} expressions, {sum(c['refused'] for c in out)} refused")


if __name__ == "__main__":
    sys.exit(main())
