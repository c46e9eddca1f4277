"""The initial condition of a reference case file, evaluated on the host into the state a run starts from.

A case file's [initial] table (cpp/include/fv/CaseFile.hpp:16-37, evaluate_initial in cpp/src/CaseFile.cpp:784-841):
a background `state` of primitive values (rho, u, v, p, w), then [[initial.region]] entries in order, each overriding
some of them where the cell centre lies inside (a box between `min` and `max`, a halfspace with (c - point) . normal >= 0,
a sphere or a cylinder along `axis` with `center` and `radius`; in 2-D only x and y count). Values are numbers or
expressions of the cell centre (x, y, z), pi, e and the run's numeric parameters (Lx, gamma, u_in, ...); region geometry
may use the parameters but not x, y, z. Primitive values missing from every table are 0. The cells are then converted
with EOS::prim_to_cons (cpp/include/fv/Core.hpp:209-221).

The reference evaluates expressions with TinyExpr (its vendored cpp/third_party/tinyexpr, compiled with
TE_POW_FROM_RIGHT: `^` is a right-associative power, `log` is the base-10 logarithm, `ln` the natural one). Here the
library's own compiler of that grammar evaluates them on the host (fvg_expr_eval, over all cells at once), with the C
library's functions the reference calls: the initial states carry the reference's bits. A value that is a whole number
is read exactly, as the reference's Evaluator does. A built-in `profile` (a C++ initialiser of the reference) is
refused: the states of the configurations' profiles are in fenice_b200.initial.
"""
import math
import tomllib

import numpy as np

from . import params as P
from .runtime import eval_expression

_STATE = {"rho": 0, "u": 1, "v": 2, "p": 3, "w": 4}   # the primitive layout [rho, u, v, p, w]


def _number(v):
    if isinstance(v, bool):
        return None
    try:
        return float(v)
    except (TypeError, ValueError):
        return None


class Expr:
    """One value of a case file: a number, or an expression evaluated by the library over arrays of cell centres.
    `names`: the (name, value) pairs bound besides x, y, z, t."""

    def __init__(self, src, names, what):
        self.src = str(src)
        self.constant = _number(src)
        self.what = what
        self.names = list(names)
        if self.constant is None:
            self([0.0], [0.0], [0.0])   # a malformed expression raises now

    def __call__(self, x, y, z):
        if self.constant is not None:
            return self.constant
        n = max(np.size(x), np.size(y), np.size(z))
        try:
            return eval_expression(self.src, self.names, np.broadcast_to(x, (n,)), np.broadcast_to(y, (n,)), np.broadcast_to(z, (n,)), 0.0)
        except ValueError as e:
            raise ValueError(f"{self.what}: {e}") from None


def _numeric_params(params):
    return [(k, n) for k, n in ((k, _number(v)) for k, v in params.items()) if n is not None and k not in ("x", "y", "z", "t")]


def _vec(exprs, fill):
    out = [fill, fill, fill]
    for d, e in enumerate(exprs):
        out[d] = float(np.asarray(e(0.0, 0.0, 0.0)).reshape(-1)[0])
    return out


def read(path):
    """The case file's parameters (flattened, as params.load_case) and its [initial] table."""
    with open(path, "rb") as f:
        doc = tomllib.load(f)
    return doc


def initial_state(initial, params, three_d_case=False):
    """The state (cells of 5 doubles, the reference's cell order) of an [initial] table for the run of `params`. A case that
    is not 3-D ([case] requires_3d) on a 3-D mesh is evaluated on one layer of the 2-D mesh (z = 0, Lz = 1, nz = 1) and
    extruded along z (Simulation::initial_field, cpp/src/Simulation.cpp:773-786)."""
    p = P.resolve(params)
    if initial.get("profile"):
        raise ValueError(f"the built-in profile '{initial['profile']}' is the reference's C++ initialiser: use fenice_b200.initial")
    if int(p["nz"]) > 1 and not three_d_case:
        layer = initial_state(initial, dict(p, nz=1, Lz=1.0), False)
        return np.tile(layer, (int(p["nz"]), 1))
    if three_d_case and int(p["nz"]) <= 1:
        raise ValueError("the case is 3-D: set nz > 1")
    nx, ny, nz = int(p["nx"]), int(p["ny"]), int(p["nz"])
    Lx, Ly, Lz = float(p["Lx"]), float(p["Ly"]), float(p["Lz"])
    three_d = nz > 1
    # x, y, z, t, the numeric parameters, then the mesh's Lx .. nz (CaseFile.cpp:313-329)
    names = _numeric_params(p) + [("Lx", Lx), ("Ly", Ly), ("Lz", Lz), ("nx", float(nx)), ("ny", float(ny)), ("nz", float(nz))]
    dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = [(i.ravel() + 0.5) * dx + 0.0, (j.ravel() + 0.5) * dy + 0.0, (k.ravel() + 0.5) * dz + 0.0 if three_d else np.zeros(i.size)]
    n = nx * ny * nz
    W = np.zeros((n, 5))
    for var, src in (initial.get("state") or {}).items():
        W[:, _STATE[var]] = Expr(src, names, f"initial.state.{var}")(*c)
    inf = math.inf
    dims = 3 if three_d else 2
    for r_i, r in enumerate(initial.get("region") or []):
        what = f"region {r_i + 1}"
        shape = r.get("shape")
        if shape == "box":
            a = _vec([Expr(v, names, what + ".min") for v in r.get("min", [])], -inf)
            b = _vec([Expr(v, names, what + ".max") for v in r.get("max", [])], inf)
            inside = np.ones(n, dtype=bool)
            for d in range(dims):
                inside &= ~((c[d] < a[d]) | (c[d] > b[d]))
        elif shape == "halfspace":
            a = _vec([Expr(v, names, what + ".point") for v in r.get("point", [])], 0.0)
            b = _vec([Expr(v, names, what + ".normal") for v in r.get("normal", [])], 0.0)
            dot = np.zeros(n)
            for d in range(dims):
                dot = dot + (c[d] - a[d]) * b[d]
            inside = dot >= 0.0
        elif shape in ("sphere", "cylinder"):
            if shape == "sphere" and three_d and len(r.get("center", [])) < 3:
                raise ValueError(f"{what}: a sphere on a 3-D mesh needs a 3-component center")
            a = _vec([Expr(v, names, what + ".center") for v in r.get("center", [])], 0.0)
            rad = float(np.asarray(Expr(r.get("radius"), names, what + ".radius")(0.0, 0.0, 0.0)).reshape(-1)[0])
            ax = {"x": 0, "y": 1, "z": 2}[r.get("axis", "z")] if shape == "cylinder" else -1
            s2 = np.zeros(n)
            for d in range(dims):
                if d != ax:
                    s2 = s2 + (c[d] - a[d]) * (c[d] - a[d])
            inside = s2 <= rad * rad
        else:
            raise ValueError(f"{what}: shape must be box, halfspace, sphere or cylinder; got '{shape}'")
        for var, src in (r.get("state") or {}).items():
            vals = Expr(src, names, f"{what}.state.{var}")(*c)
            W[:, _STATE[var]] = np.where(inside, vals, W[:, _STATE[var]])
    return prim_to_cons(W, float(p["gamma"]), float(p["p_inf"]), str(p["eos_type"]).strip().lower() != "ideal gas")


def prim_to_cons(W, gamma, p_inf=0.0, stiffened=False):
    """EOS::prim_to_cons (Core.hpp:209-221) of cells [rho, u, v, p, w]."""
    r, u, v, p, w = W[:, 0], W[:, 1], W[:, 2], W[:, 3], W[:, 4]
    U = np.empty_like(W)
    ke = 0.5 * r * (u * u + v * v + w * w)
    e = (p + gamma * p_inf) / (gamma - 1.0) if stiffened else p / (gamma - 1.0)
    U[:, 0] = r
    U[:, 1] = r * u
    U[:, 2] = r * v
    U[:, 3] = e + ke
    U[:, 4] = r * w
    return U


def load(path, overrides=None):
    """(params, U0) of a case file: its parameters with `overrides` on top, and its initial state on that mesh."""
    params, initial = P.load_case(path, overrides)
    three_d = bool(read(path).get("case", {}).get("requires_3d", False))
    return params, initial_state(initial, params, three_d)
