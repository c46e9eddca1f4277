"""The reference's run parameters and case files, turned into the C ABI's fvg_config.

A run is described with the reference's own parameter keys (its case-file / ``--set`` keys, cpp/src/Params.cpp:100-160)
and values, e.g. ``{"nx": 256, "reconstruction": "weno5", "riemann_solver": "HLLC (Low-Mach Thornber)"}``; missing keys
take the reference's defaults. Names are parsed as the reference parses them (case-insensitive, GUI labels and aliases:
parse_riemann / parse_limiter / parse_reconstruction, cpp/src/Schemes.cpp:77-102; parse_bc,
cpp/src/Boundaries.cpp:15-27; parse_time_scheme, cpp/src/TimeScheme.cpp:73-80) and an unknown name raises ValueError,
as the reference raises std::invalid_argument. ``time_scheme = "auto"`` resolves as in SimParams::from
(cpp/src/Params.cpp:360-363), and boundary_order 2 falls back to 1 without a reconstruction (Params.cpp:470).
"""
import ctypes
import tomllib

from . import airfoil

DEFAULTS = {
    "Lx": 1.0, "Ly": 1.0, "Lz": 1.0, "nx": 100, "ny": 100, "nz": 1,
    "eos_type": "Ideal Gas", "gamma": 1.4, "p_inf": 0.0,
    "use_viscous": False, "mu": 1e-3, "pr": 0.72,
    "bc_xmin": "wall", "bc_xmax": "wall", "bc_ymin": "wall", "bc_ymax": "wall", "bc_zmin": "periodic", "bc_zmax": "periodic",
    "u_in": 0.0, "v_in": 0.0, "rho_in": 1.0, "p_out": 1.0,
    "riemann_solver": "HLLC", "reconstruction": "none", "muscl_limiter": "Van Leer", "weno_epsilon": 1e-6,
    "boundary_order": 2, "time_scheme": "auto", "cfl": 0.5, "shock_blend": 0.2, "dt_max": 0.0, "t_end": 0.005,
    "max_steps": 0,
    "use_ibm": False, "ibm_shape": "Cylinder", "ibm_radius": 0.1, "ibm_cx": 0.5, "ibm_cy": 0.5, "ibm_cz": 0.5, "ibm_curvature": False,
    "use_bodyforce": False, "gx": 0.0, "gy": -9.81, "gz": 0.0, "nrbc_sigma": 0.28, "nrbc_beta": -1.0, "positivity_fallback": False,
}

BC_NAMES = {"wall": 0, "inviscid wall (slip)": 0, "no_slip": 1, "viscous wall (no-slip)": 1, "moving_wall": 2, "moving wall": 2,
            "vel_inlet": 3, "velocity inlet": 3, "massflow_inlet": 4, "mass flow inlet": 4, "outlet": 5, "pressure outlet": 5,
            "transmissive": 6, "periodic": 7, "nonreflecting": 8, "non_reflecting": 8, "non-reflecting outlet": 8}
RIEMANN_NAMES = {"hllc": 0, "hllc (low-mach thornber)": 1, "lowmach": 1, "lowmachhllc": 1, "low-mach": 1}
RECON_NAMES = {"none": 0, "muscl": 1, "weno3": 2, "weno5": 3}
LIMITER_NAMES = {"minmod": 0, "van leer": 1, "vanleer": 1, "mc": 2, "koren": 3}
SCHEME_NAMES = {"explicit euler": 0, "euler": 0, "explicit_euler": 0, "ssp runge-kutta 2": 1, "ssprk2": 1, "rk2": 1,
                "ssp runge-kutta 3": 2, "ssprk3": 2, "rk3": 2, "muscl-hancock": 3, "hancock": 3}
STAGES = {0: 1, 1: 2, 2: 3, 3: 1}   # residual evaluations per step (MUSCL-Hancock: one, after its first step)


class FvgConfig(ctypes.Structure):
    """struct fvg_config of include/fenice_gpu.h"""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
                ("eos_type", ctypes.c_int), ("gamma", ctypes.c_double), ("p_inf", ctypes.c_double),
                ("bc", ctypes.c_int * 6), ("u_in", ctypes.c_double), ("v_in", ctypes.c_double),
                ("rho_in", ctypes.c_double), ("p_out", ctypes.c_double),
                ("riemann", ctypes.c_int), ("shock_blend", ctypes.c_double),
                ("reconstruction", ctypes.c_int), ("limiter", ctypes.c_int), ("weno_epsilon", ctypes.c_double),
                ("boundary_order", ctypes.c_int), ("time_scheme", ctypes.c_int),
                ("cfl", ctypes.c_double), ("dt_max", ctypes.c_double),
                ("use_viscous", ctypes.c_int), ("mu", ctypes.c_double), ("pr", ctypes.c_double),
                ("precision", ctypes.c_int), ("device", ctypes.c_int),
                ("use_ibm", ctypes.c_int), ("ibm_shape", ctypes.c_int), ("ibm_radius", ctypes.c_double), ("ibm_cx", ctypes.c_double),
                ("ibm_cy", ctypes.c_double), ("ibm_cz", ctypes.c_double), ("ibm_curvature", ctypes.c_int),
                ("use_bodyforce", ctypes.c_int), ("gx", ctypes.c_double), ("gy", ctypes.c_double), ("gz", ctypes.c_double),
                ("nrbc_sigma", ctypes.c_double), ("nrbc_beta", ctypes.c_double), ("positivity_fallback", ctypes.c_int),
                ("source", ctypes.c_char_p * 5), ("boundary_expr", ctypes.c_char_p * 4),
                ("boundary_table", ctypes.POINTER(ctypes.c_double) * 4), ("boundary_table_rows", ctypes.c_int * 4),
                ("param_names", ctypes.POINTER(ctypes.c_char_p)), ("param_values", ctypes.POINTER(ctypes.c_double)), ("nparams", ctypes.c_int),
                ("flux_quadrature", ctypes.c_int),
                ("ibm_vx", ctypes.c_double), ("ibm_vy", ctypes.c_double), ("ibm_vz", ctypes.c_double),
                ("ibm_omega", ctypes.c_double), ("ibm_omega_x", ctypes.c_double), ("ibm_omega_y", ctypes.c_double),
                ("ibm_omega_from", ctypes.c_double), ("ibm_omega_until", ctypes.c_double),
                ("ibm_mass", ctypes.c_double), ("ibm_inertia", ctypes.c_double),
                ("ibm_stiff_x", ctypes.c_double), ("ibm_stiff_y", ctypes.c_double), ("ibm_stiff_z", ctypes.c_double),
                ("ibm_damp_x", ctypes.c_double), ("ibm_damp_y", ctypes.c_double), ("ibm_damp_z", ctypes.c_double),
                ("ibm_stiff_theta", ctypes.c_double), ("ibm_damp_theta", ctypes.c_double),
                ("ibm_cm_x", ctypes.c_double), ("ibm_cm_y", ctypes.c_double), ("ibm_cm_given", ctypes.c_int),
                ("ibm_section", ctypes.POINTER(ctypes.c_double)), ("ibm_section_points", ctypes.c_int),
                ("ibm_chord", ctypes.c_double), ("ibm_aoa", ctypes.c_double)]

BODY_KEYS = ("ibm_vx", "ibm_vy", "ibm_vz", "ibm_omega", "ibm_omega_x", "ibm_omega_y", "ibm_omega_from", "ibm_omega_until", "ibm_mass",
             "ibm_inertia", "ibm_stiff_x", "ibm_stiff_y", "ibm_stiff_z", "ibm_damp_x", "ibm_damp_y", "ibm_damp_z", "ibm_stiff_theta",
             "ibm_damp_theta")

SOURCE_KEYS = ("source_rho", "source_mx", "source_my", "source_E", "source_mz")   # the state's slot order
BOUNDARY_KEYS = ("u_in", "v_in", "rho_in", "p_out")


def _flag(v):
    if isinstance(v, str):
        s = v.strip().lower()
        if s in ("1", "true", "yes", "on"):
            return True
        if s in ("0", "false", "no", "off", ""):
            return False
        raise ValueError(f"not a boolean: {v!r}")
    return bool(v)


def _pick(table, value, what):
    key = str(value).strip().lower()
    if key not in table:
        raise ValueError(f"Unknown {what}: '{value}'")
    return table[key]


def resolve(params):
    """The parameters with the reference's defaults filled in and time_scheme = auto resolved."""
    p = dict(DEFAULTS)
    p.update(params)
    if str(p["time_scheme"]).strip().lower() == "auto":
        rec = str(p["reconstruction"]).strip().lower()
        p["time_scheme"] = "Explicit Euler" if rec != "muscl" else ("SSP Runge-Kutta 2" if _flag(p["use_viscous"]) else "MUSCL-Hancock")
    # a first-order run keeps first-order boundaries (Params.cpp:470)
    if int(p["boundary_order"]) == 2 and str(p["reconstruction"]).strip().lower() == "none":
        p["boundary_order"] = 1
    return p


def _num(v):
    try:
        return float(v)
    except (TypeError, ValueError):
        return None


def not_on_device(params):
    """The reference features a parameter dict switches on that the device path does not compute (None: none). They
    are refused, never ignored: AMR. (Combinations
    the device refuses, such as the body force with the mixed-precision form, are refused by fvg_create with
    FVG_ERR_CONFIG.)"""
    p = resolve(params)
    if _flag(p.get("use_amr", False)):
        return "adaptive meshes (use_amr)"
    return None


def read_time_table(path):
    """The rows (t, value) of a boundary time table (read_time_table, cpp/src/SimulationInternal.hpp:62-99): one row per
    line, comma- or space-separated, '#' comments and blank lines skipped, an optional 't,value' / 'time,value' header
    before the first row, a UTF-8 byte-order mark dropped; finite values, strictly increasing times, at least two rows."""
    rows = []
    with open(path, "rb") as f:
        text = f.read()
    if text.startswith(b"\xef\xbb\xbf"):
        text = text[3:]
    for n, raw in enumerate(text.decode().split("\n"), 1):
        line = raw.strip(" \t\r")
        if not line or line.startswith("#"):
            continue
        parts = line.replace(",", " ").split()
        try:
            t, v = float(parts[0]), float(parts[1])
        except (ValueError, IndexError):
            if not rows and len(parts) == 2 and parts[0].lower() in ("t", "time") and parts[1].lower() == "value":
                continue
            raise ValueError(f"{path}:{n} must contain t,value") from None
        if len(parts) > 2:
            raise ValueError(f"{path}:{n} has more than two columns")
        if not (abs(t) < float("inf") and abs(v) < float("inf")):
            raise ValueError(f"{path}:{n} values must be finite")
        if rows and not t > rows[-1][0]:
            raise ValueError(f"{path}: times must be strictly increasing")
        rows.append((t, v))
    if len(rows) < 2:
        raise ValueError(f"{path} must contain at least two (t,value) rows")
    return rows


def _bound_names(p):
    """The names the reference's Evaluator binds besides x, y, z, t: every numeric run parameter (Lx .. nz are bound again
    from the mesh by the library)."""
    out = []
    for k, v in p.items():
        if k in ("x", "y", "z", "t") or isinstance(v, bool):
            continue
        n = _num(v)
        if n is not None:
            out.append((str(k), n))
    return out


def _initial_boundary_value(p, key):
    """u_in / v_in / rho_in / p_out at t = 0 (load_boundary_functions, cpp/src/Simulation.cpp:145-153)."""
    table = str(p.get(key + "_table", "") or "").strip()
    if table:
        return read_time_table(table)[0][1]
    v = _num(p[key])
    if v is not None:
        return v
    from .runtime import eval_expression

    return float(eval_expression(str(p[key]), _bound_names(p) + [(k, float(p[k])) for k in ("Lx", "Ly", "Lz", "nx", "ny", "nz")], [0.0], [0.0], [0.0], 0.0)[0])


def to_config(params, precision=0, device=0):
    """fvg_config of a parameter dict (reference keys); ValueError for a feature the device path does not compute."""
    why = not_on_device(params)
    if why:
        raise ValueError(f"not computed by the device path: {why}")
    p = resolve(params)
    c = FvgConfig()
    c.nx, c.ny, c.nz = int(p["nx"]), int(p["ny"]), int(p["nz"])
    c.Lx, c.Ly, c.Lz = float(p["Lx"]), float(p["Ly"]), float(p["Lz"])
    c.eos_type = 0 if str(p["eos_type"]).strip().lower() == "ideal gas" else 1
    c.gamma, c.p_inf = float(p["gamma"]), float(p["p_inf"])
    for s, key in enumerate(("bc_xmin", "bc_xmax", "bc_ymin", "bc_ymax", "bc_zmin", "bc_zmax")):
        c.bc[s] = _pick(BC_NAMES, p[key], "boundary condition type")
    # u_in, v_in, rho_in, p_out: numbers, expressions of t or time tables (load_boundary_functions, Simulation.cpp:118-168)
    keep = []
    for k, key in enumerate(BOUNDARY_KEYS):
        v = _num(p[key])
        setattr(c, key, v if v is not None else (1.0 if key in ("rho_in", "p_out") else 0.0))
        if v is None:
            c.boundary_expr[k] = str(p[key]).encode()
        table = str(p.get(key + "_table", "") or "").strip()
        if table:
            if v is None:
                raise ValueError(f"{key} expression and {key}_table cannot both be set")
            rows = (ctypes.c_double * (2 * len(read_time_table(table))))(*[x for r in read_time_table(table) for x in r])
            keep.append(rows)
            c.boundary_table[k] = ctypes.cast(rows, ctypes.POINTER(ctypes.c_double))
            c.boundary_table_rows[k] = len(rows) // 2
    # reynolds > 0: mu from the body's length scale and the inflow at t = 0 (Simulation.cpp:154-167)
    if (_num(p.get("reynolds", 0)) or 0.0) > 0.0:
        rho0, u0 = _initial_boundary_value(p, "rho_in"), _initial_boundary_value(p, "u_in")
        if not (rho0 > 0.0 and u0 > 0.0):
            raise ValueError("reynolds needs positive u_in and rho_in at t=0 (including boundary tables)")
        p = dict(p, mu=rho0 * u0 * (2.0 * float(p["ibm_radius"])) / float(p["reynolds"]))
    for q, key in enumerate(SOURCE_KEYS):
        c.source[q] = str(p.get(key, "0")).encode()
    names = _bound_names(p)
    c.nparams = len(names)
    if names:
        cn = (ctypes.c_char_p * len(names))(*[k.encode() for k, _ in names])
        cv = (ctypes.c_double * len(names))(*[v for _, v in names])
        keep += [cn, cv]
        c.param_names = ctypes.cast(cn, ctypes.POINTER(ctypes.c_char_p))
        c.param_values = ctypes.cast(cv, ctypes.POINTER(ctypes.c_double))
    c._keep = keep   # the arrays the pointers above point into live as long as the configuration
    c.riemann = _pick(RIEMANN_NAMES, p["riemann_solver"], "Riemann solver")
    c.shock_blend = float(p["shock_blend"])
    c.reconstruction = _pick(RECON_NAMES, p["reconstruction"], "reconstruction")
    c.limiter = _pick(LIMITER_NAMES, p["muscl_limiter"], "MUSCL limiter")
    c.weno_epsilon = float(p["weno_epsilon"])
    c.boundary_order = int(p["boundary_order"])
    c.time_scheme = _pick(SCHEME_NAMES, p["time_scheme"], "time scheme")
    c.cfl, c.dt_max = float(p["cfl"]), float(p["dt_max"])
    c.use_viscous = 1 if _flag(p["use_viscous"]) else 0
    c.mu, c.pr = float(p["mu"]), float(p["pr"])
    c.precision = int(precision)
    c.device = int(device)
    c.use_ibm = 1 if _flag(p["use_ibm"]) else 0
    shape = str(p["ibm_shape"]).strip().lower()
    digits = airfoil.naca_digits(p["ibm_shape"])
    if shape not in ("cylinder", "sphere", "airfoil") and not digits:   # Params.cpp:497-501
        raise ValueError(f"Unknown ibm_shape: '{p['ibm_shape']}' (use Cylinder, Sphere, Airfoil or NACA dddd)")
    c.ibm_shape = 1 if shape == "sphere" else (2 if (shape == "airfoil" or digits) else 0)
    c.ibm_chord, c.ibm_aoa = float(p.get("ibm_chord", 1.0)), float(p.get("ibm_aoa", 0.0))
    if c.use_ibm and c.ibm_shape == 2:   # the unit section: a NACA 4-digit one, or a coordinate file (ibm_file)
        if digits:
            section = airfoil.naca4(digits)
        else:
            path = str(p.get("ibm_file", "") or "").strip()
            if not path:
                raise ValueError("ibm_shape = Airfoil needs ibm_file (a Selig or Lednicer coordinate file)")
            section = airfoil.load_airfoil(path)
        arr = (ctypes.c_double * (2 * len(section)))(*[v for q in section for v in q])
        c._section = arr
        c.ibm_section = ctypes.cast(arr, ctypes.POINTER(ctypes.c_double))
        c.ibm_section_points = len(section)
    c.ibm_radius, c.ibm_cx, c.ibm_cy, c.ibm_cz = float(p["ibm_radius"]), float(p["ibm_cx"]), float(p["ibm_cy"]), float(p["ibm_cz"])
    c.ibm_curvature = 1 if _flag(p["ibm_curvature"]) else 0
    c.use_bodyforce = 1 if _flag(p["use_bodyforce"]) else 0
    c.gx, c.gy, c.gz = float(p["gx"]), float(p["gy"]), float(p["gz"])
    c.nrbc_sigma, c.nrbc_beta = float(p["nrbc_sigma"]), float(p["nrbc_beta"])
    c.positivity_fallback = 1 if _flag(p["positivity_fallback"]) else 0
    quad = str(p.get("flux_quadrature", "midpoint")).strip().lower()
    if quad not in ("midpoint", "fourth"):   # Params.cpp:448-449
        raise ValueError(f"flux_quadrature must be midpoint or fourth; got '{quad}'")
    c.flux_quadrature = 1 if quad == "fourth" else 0
    c.mu = float(p["mu"])   # (derived from reynolds above when given)
    for k in BODY_KEYS:
        setattr(c, k, float(p.get(k, 0.0)) if c.use_ibm else 0.0)
    # the centre of mass off the pivot: both keys given (Params.cpp:334-338)
    cmx, cmy = str(p.get("ibm_cm_x", "")).strip(), str(p.get("ibm_cm_y", "")).strip()
    if bool(cmx) != bool(cmy):
        raise ValueError("ibm_cm_x and ibm_cm_y go together")
    c.ibm_cm_given = 1 if (cmx and cmy and c.use_ibm) else 0
    c.ibm_cm_x, c.ibm_cm_y = (float(cmx), float(cmy)) if c.ibm_cm_given else (0.0, 0.0)
    return c


def load_case(path, overrides=None):
    """The parameters of a reference case file (TOML, sections [mesh] [thermo] [physics] [boundaries] [numerics] [run] ...;
    cpp/include/fv/CaseFile.hpp:19-37), flattened to keys, with `overrides` on top. The [initial] table is returned
    separately (the initial condition is the caller's: a state array)."""
    with open(path, "rb") as f:
        doc = tomllib.load(f)
    params = {}
    for section, table in doc.items():
        if section in ("case", "initial") or not isinstance(table, dict):
            continue
        for k, v in table.items():
            if not isinstance(v, (dict, list)):
                params[k] = v
    params.update(overrides or {})
    # a boundary time table is looked for next to the case file, then in the current folder (Simulation.cpp:128-139)
    import os

    for k, v in list(params.items()):
        if (k.endswith("_table") or k == "ibm_file") and isinstance(v, str) and v.strip() and not os.path.isabs(v.strip()):
            beside = os.path.join(os.path.dirname(os.path.abspath(path)), v.strip())
            if os.path.exists(beside):
                params[k] = beside
    return params, doc.get("initial", {})
