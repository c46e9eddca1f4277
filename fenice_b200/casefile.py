"""The initial condition of a reference case file, evaluated on the host into the state a run starts from.

A case file's [initial] table (cpp/include/fv/CaseFile.hpp:16-37, evaluate_initial in cpp/src/CaseFile.cpp:784-841):
a background `state` of primitive values (rho, u, v, p, w), then [[initial.region]] entries in order, each overriding
some of them where the cell centre lies inside (a box between `min` and `max`, a halfspace with (c - point) . normal >= 0,
a sphere or a cylinder along `axis` with `center` and `radius`; in 2-D only x and y count). Values are numbers or
expressions of the cell centre (x, y, z), pi, e and the run's numeric parameters (Lx, gamma, u_in, ...); region geometry
may use the parameters but not x, y, z. Primitive values missing from every table are 0. The cells are then converted
with EOS::prim_to_cons (cpp/include/fv/Core.hpp:209-221).

The reference evaluates expressions with TinyExpr (its vendored cpp/third_party/tinyexpr, compiled with
TE_POW_FROM_RIGHT: `^` is a right-associative power, `log` is the base-10 logarithm, `ln` the natural one). The same
grammar is evaluated here, vectorised over the cells with numpy: + - * / % ^, unary minus, parentheses, the names above
and sin cos tan asin acos atan atan2 sinh cosh tanh exp sqrt pow abs ln log log10 ceil floor. Numbers, arithmetic and
geometry give the reference's bits; numpy's transcendental functions may differ from the C library's by an ulp. A
built-in `profile` (a C++ initialiser of the reference) is refused: the states of the configurations' profiles are in
fenice_b200.initial.
"""
import ast
import math
import tomllib

import numpy as np

from . import params as P

_FUNCS = {"sin": np.sin, "cos": np.cos, "tan": np.tan, "asin": np.arcsin, "acos": np.arccos, "atan": np.arctan, "atan2": np.arctan2,
          "sinh": np.sinh, "cosh": np.cosh, "tanh": np.tanh, "exp": np.exp, "sqrt": np.sqrt, "pow": np.power, "abs": np.abs, "ln": np.log,
          "log": np.log10, "log10": np.log10, "ceil": np.ceil, "floor": np.floor}
_CONSTS = {"pi": math.pi, "e": math.e}
_BINOPS = {ast.Add: np.add, ast.Sub: np.subtract, ast.Mult: np.multiply, ast.Div: np.divide, ast.Pow: np.power, ast.Mod: np.fmod}
_STATE = {"rho": 0, "u": 1, "v": 2, "p": 3, "w": 4}   # the primitive layout [rho, u, v, p, w]


def _number(v):
    try:
        return float(v)
    except (TypeError, ValueError):
        return None


class Expr:
    """One value of a case file: a number, or an expression compiled once and evaluated over arrays of cell centres."""

    def __init__(self, src, names, what):
        self.src = str(src)
        self.constant = _number(src) if not isinstance(src, bool) else None
        self.what = what
        if self.constant is not None:
            return
        try:
            tree = ast.parse(self.src.replace("^", "**"), mode="eval")
        except SyntaxError as e:
            raise ValueError(f"{what}: cannot evaluate \"{self.src}\" ({e.msg})") from None
        self._check(tree.body, names)
        self.tree = tree.body

    def _check(self, node, names):
        if isinstance(node, ast.BinOp) and type(node.op) in _BINOPS:
            self._check(node.left, names)
            self._check(node.right, names)
        elif isinstance(node, ast.UnaryOp) and isinstance(node.op, (ast.USub, ast.UAdd)):
            self._check(node.operand, names)
        elif isinstance(node, ast.Constant) and isinstance(node.value, (int, float)) and not isinstance(node.value, bool):
            pass
        elif isinstance(node, ast.Name):
            if node.id not in names and node.id not in _CONSTS:
                raise ValueError(f"{self.what}: unknown name '{node.id}' in \"{self.src}\"")
        elif isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id in _FUNCS and not node.keywords:
            for a in node.args:
                self._check(a, names)
        else:
            raise ValueError(f"{self.what}: \"{self.src}\" is not an expression of numbers, names, + - * / % ^ and functions")

    def __call__(self, env):
        if self.constant is not None:
            return self.constant
        return self._eval(self.tree, env)

    def _eval(self, node, env):
        if isinstance(node, ast.BinOp):
            return _BINOPS[type(node.op)](self._eval(node.left, env), self._eval(node.right, env))
        if isinstance(node, ast.UnaryOp):
            v = self._eval(node.operand, env)
            return np.negative(v) if isinstance(node.op, ast.USub) else v
        if isinstance(node, ast.Constant):
            return float(node.value)
        if isinstance(node, ast.Name):
            return env[node.id] if node.id in env else _CONSTS[node.id]
        return _FUNCS[node.func.id](*[self._eval(a, env) for a in node.args])


def _numeric_params(params):
    env = {}
    for k, v in params.items():
        n = _number(v) if not isinstance(v, bool) else None
        if n is not None:
            env[k] = n
    return env


def _vec(exprs, env, fill):
    out = [fill, fill, fill]
    for d, e in enumerate(exprs):
        out[d] = float(e(env))
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
    env = _numeric_params(p)
    env.update(Lx=Lx, Ly=Ly, Lz=Lz, nx=float(nx), ny=float(ny), nz=float(nz), t=0.0)
    names = set(env) | {"x", "y", "z"}
    dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cell = {"x": ((i.ravel() + 0.5) * dx + 0.0), "y": ((j.ravel() + 0.5) * dy + 0.0), "z": ((k.ravel() + 0.5) * dz + 0.0) if three_d else
            np.zeros(i.size)}
    genv = dict(env, x=0.0, y=0.0, z=0.0)
    cenv = dict(env, **cell)
    n = nx * ny * nz
    W = np.zeros((n, 5))
    for var, src in (initial.get("state") or {}).items():
        W[:, _STATE[var]] = Expr(src, names, f"initial.state.{var}")(cenv)
    inf = math.inf
    dims = 3 if three_d else 2
    c = [cell["x"], cell["y"], cell["z"]]
    for r_i, r in enumerate(initial.get("region") or []):
        what = f"region {r_i + 1}"
        shape = r.get("shape")
        if shape == "box":
            a = _vec([Expr(v, names, what + ".min") for v in r.get("min", [])], genv, -inf)
            b = _vec([Expr(v, names, what + ".max") for v in r.get("max", [])], genv, inf)
            inside = np.ones(n, dtype=bool)
            for d in range(dims):
                inside &= ~((c[d] < a[d]) | (c[d] > b[d]))
        elif shape == "halfspace":
            a = _vec([Expr(v, names, what + ".point") for v in r.get("point", [])], genv, 0.0)
            b = _vec([Expr(v, names, what + ".normal") for v in r.get("normal", [])], genv, 0.0)
            dot = np.zeros(n)
            for d in range(dims):
                dot = dot + (c[d] - a[d]) * b[d]
            inside = dot >= 0.0
        elif shape in ("sphere", "cylinder"):
            if shape == "sphere" and three_d and len(r.get("center", [])) < 3:
                raise ValueError(f"{what}: a sphere on a 3-D mesh needs a 3-component center")
            a = _vec([Expr(v, names, what + ".center") for v in r.get("center", [])], genv, 0.0)
            rad = float(Expr(r.get("radius"), names, what + ".radius")(genv))
            ax = {"x": 0, "y": 1, "z": 2}[r.get("axis", "z")] if shape == "cylinder" else -1
            s = np.zeros(n)
            for d in range(dims):
                if d != ax:
                    s = s + (c[d] - a[d]) * (c[d] - a[d])
            inside = s <= rad * rad
        else:
            raise ValueError(f"{what}: shape must be box, halfspace, sphere or cylinder; got '{shape}'")
        for var, src in (r.get("state") or {}).items():
            vals = Expr(src, names, f"{what}.state.{var}")(cenv)
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
