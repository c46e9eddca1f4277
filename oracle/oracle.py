"""ctypes access to the two CPU checkers of the CUDA path (TEST INFRASTRUCTURE: imported only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg; the product never imports it).

* ``Oracle``: the C restatement of the reference path, oracle/liboracle.so (oracle/fv_oracle.c).
* ``Reference``: the reference solver itself, compiled from its own sources into oracle/_ref/ by
  oracle/ref/Makefile, driven through the extern "C" harness oracle/ref/ref_harness.cpp.

Both take a run as a dict of the reference's own parameter keys (its case-file / ``--set`` keys: nx, ny, nz,
Lx, Ly, Lz, eos_type, gamma, p_inf, bc_xmin .. bc_zmax, u_in, v_in, rho_in, p_out, riemann_solver,
shock_blend, reconstruction, muscl_limiter, weno_epsilon, boundary_order, time_scheme, cfl, dt_max,
use_viscous, mu, pr) and states as (ncells, 5) float64 arrays in the reference's layout
[rho, rho u, rho v, rho E, rho w], cell (k*ny + j)*nx + i.
"""
import contextlib
import ctypes
import os
import sys

import numpy as np


@contextlib.contextmanager
def quiet_stdout():
    """The reference prints progress lines on its setup; keep them off this process's stdout (fd 1)."""
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    try:
        os.dup2(devnull, 1)
        yield
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfenice_ref.so")

# defaults of the reference's parameter table (cpp/src/Params.cpp:100-160)
DEFAULTS = {
    "Lx": 1.0, "Ly": 1.0, "Lz": 1.0, "nx": 100, "ny": 100, "nz": 1,
    "eos_type": "Ideal Gas", "gamma": 1.4, "p_inf": 0.0,
    "use_viscous": False, "mu": 1e-3, "pr": 0.72,
    "bc_xmin": "wall", "bc_xmax": "wall", "bc_ymin": "wall", "bc_ymax": "wall", "bc_zmin": "periodic", "bc_zmax": "periodic",
    "u_in": 0.0, "v_in": 0.0, "rho_in": 1.0, "p_out": 1.0,
    "riemann_solver": "HLLC", "reconstruction": "none", "muscl_limiter": "Van Leer", "weno_epsilon": 1e-6,
    "boundary_order": 2, "time_scheme": "auto", "cfl": 0.5, "shock_blend": 0.2, "dt_max": 0.0,
}

_BC = {"wall": 0, "inviscid wall (slip)": 0, "no_slip": 1, "viscous wall (no-slip)": 1, "moving_wall": 2, "moving wall": 2,
       "vel_inlet": 3, "velocity inlet": 3, "massflow_inlet": 4, "mass flow inlet": 4, "outlet": 5, "pressure outlet": 5,
       "transmissive": 6, "periodic": 7, "nonreflecting": 8, "non_reflecting": 8, "non-reflecting outlet": 8}
_RIEMANN = {"hllc": 0, "hllc (low-mach thornber)": 1, "lowmach": 1, "lowmachhllc": 1, "low-mach": 1}
_RECON = {"none": 0, "muscl": 1, "weno3": 2, "weno5": 3}
_LIMITER = {"minmod": 0, "van leer": 1, "vanleer": 1, "mc": 2, "koren": 3}
_SCHEME = {"explicit euler": 0, "euler": 0, "explicit_euler": 0, "ssp runge-kutta 2": 1, "ssprk2": 1, "rk2": 1,
           "ssp runge-kutta 3": 2, "ssprk3": 2, "rk3": 2, "muscl-hancock": 3, "hancock": 3}


def _flag(v):
    if isinstance(v, str):
        return v.strip().lower() in ("1", "true", "yes", "on")
    return bool(v)


def resolved(params):
    """The parameter dict with the reference's defaults filled in and time_scheme=auto resolved
    (cpp/src/Params.cpp:360-363)."""
    p = dict(DEFAULTS)
    p.update(params)
    if str(p["time_scheme"]).lower() == "auto":
        rec = str(p["reconstruction"]).lower()
        p["time_scheme"] = "Explicit Euler" if rec != "muscl" else ("SSP Runge-Kutta 2" if _flag(p["use_viscous"]) else "MUSCL-Hancock")
    return p


class OracleConfig(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
                ("eos", ctypes.c_int), ("gamma", ctypes.c_double), ("p_inf", ctypes.c_double),
                ("bc", ctypes.c_int * 6), ("u_in", ctypes.c_double), ("v_in", ctypes.c_double),
                ("rho_in", ctypes.c_double), ("p_out", ctypes.c_double),
                ("riemann", ctypes.c_int), ("shock_blend", ctypes.c_double),
                ("recon", ctypes.c_int), ("limiter", ctypes.c_int), ("weno_eps", ctypes.c_double),
                ("boundary_order", ctypes.c_int), ("time_scheme", ctypes.c_int),
                ("cfl", ctypes.c_double), ("dt_max", ctypes.c_double),
                ("viscous", ctypes.c_int), ("mu", ctypes.c_double), ("pr", ctypes.c_double)]


def not_covered(p):
    """Features the restatement does not compute (it refuses them rather than ignore them)."""
    if _flag(p.get("use_ibm", False)):
        return "the immersed body"
    if _flag(p.get("use_bodyforce", False)):
        return "the body force"
    for k in ("source_rho", "source_mx", "source_my", "source_mz", "source_E"):
        try:
            if float(p.get(k, 0)) != 0.0:
                return "source terms"
        except (TypeError, ValueError):
            return "source terms"
    if _flag(p.get("use_amr", False)) or _flag(p.get("positivity_fallback", False)):
        return "AMR / the positivity fallback"
    return None


def oracle_config(params):
    p = resolved(params)
    why = not_covered(p)
    if why:
        raise ValueError(f"the restatement does not cover {why}")
    c = OracleConfig()
    c.nx, c.ny, c.nz = int(p["nx"]), int(p["ny"]), int(p["nz"])
    c.Lx, c.Ly, c.Lz = float(p["Lx"]), float(p["Ly"]), float(p["Lz"])
    c.eos = 0 if str(p["eos_type"]).lower() == "ideal gas" else 1
    c.gamma, c.p_inf = float(p["gamma"]), float(p["p_inf"])
    for s, key in enumerate(("bc_xmin", "bc_xmax", "bc_ymin", "bc_ymax", "bc_zmin", "bc_zmax")):
        c.bc[s] = _BC[str(p[key]).lower()]
    c.u_in, c.v_in, c.rho_in, c.p_out = float(p["u_in"]), float(p["v_in"]), float(p["rho_in"]), float(p["p_out"])
    c.riemann = _RIEMANN[str(p["riemann_solver"]).lower()]
    c.shock_blend = float(p["shock_blend"])
    c.recon = _RECON[str(p["reconstruction"]).lower()]
    c.limiter = _LIMITER[str(p["muscl_limiter"]).lower()]
    c.weno_eps = float(p["weno_epsilon"])
    c.boundary_order = int(p["boundary_order"])
    c.time_scheme = _SCHEME[str(p["time_scheme"]).lower()]
    c.cfl, c.dt_max = float(p["cfl"]), float(p["dt_max"])
    c.viscous = 1 if _flag(p["use_viscous"]) else 0
    c.mu, c.pr = float(p["mu"]), float(p["pr"])
    return c


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """The C restatement (oracle/fv_oracle.c)."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"{ORACLE_SO} is not built (make -C oracle)")
        lib = ctypes.CDLL(ORACLE_SO)
        P = ctypes.POINTER
        lib.orc_residual.argtypes = [P(OracleConfig), P(ctypes.c_double), P(ctypes.c_double), ctypes.c_double, P(ctypes.c_double)]
        lib.orc_step.argtypes = [P(OracleConfig), P(ctypes.c_double), ctypes.c_double, ctypes.c_double, P(ctypes.c_double),
                                 P(ctypes.c_double), P(ctypes.c_double)]
        lib.orc_dt_length.argtypes = [P(OracleConfig)]
        lib.orc_dt_length.restype = ctypes.c_double
        lib.orc_riemann_hash.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.orc_riemann_hash.restype = ctypes.c_ulonglong
        lib.orc_riemann_pool.argtypes = [ctypes.c_int, P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_int)]
        lib.orc_face_flux.argtypes = [P(OracleConfig), P(ctypes.c_double), P(ctypes.c_double), ctypes.c_int, P(ctypes.c_double)]
        lib.orc_face_flux.restype = ctypes.c_double
        self.lib = lib

    def residual(self, params, U, predictor_half_dt=0.0):
        c = oracle_config(params)
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.zeros_like(U)
        s = ctypes.c_double(0.0)
        rc = self.lib.orc_residual(ctypes.byref(c), _dp(U), _dp(R), float(predictor_half_dt), ctypes.byref(s))
        if rc:
            raise ValueError(f"oracle residual: configuration not covered (code {rc})")
        return R, s.value

    def run(self, params, U, n_steps, t0=0.0, t_end=1e300, lagged=0.0):
        """n_steps steps of the time scheme from U at t0 (stopping at t_end); returns (U, t, dts, smaxs, lagged)."""
        c = oracle_config(params)
        U = np.array(U, dtype=np.float64, copy=True, order="C")
        t = float(t0)
        lag = ctypes.c_double(lagged)
        dts, sms = [], []
        for _ in range(n_steps):
            if not t < t_end:
                break
            dt, sm = ctypes.c_double(0.0), ctypes.c_double(0.0)
            rc = self.lib.orc_step(ctypes.byref(c), _dp(U), t, float(t_end), ctypes.byref(lag), ctypes.byref(dt), ctypes.byref(sm))
            if rc:
                raise ValueError(f"oracle step: configuration not covered (code {rc})")
            t += dt.value
            dts.append(dt.value)
            sms.append(sm.value)
        return U, t, np.array(dts), np.array(sms), lag.value

    def dt_length(self, params):
        c = oracle_config(params)
        return self.lib.orc_dt_length(ctypes.byref(c))

    def riemann_hash(self, eos_kind, riemann):
        return int(self.lib.orc_riemann_hash(int(eos_kind), int(riemann)))

    def riemann_pool(self, eos_kind):
        n = 1 << 16
        UL = np.zeros((n, 5))
        UR = np.zeros((n, 5))
        ax = np.zeros(n, dtype=np.int32)
        self.lib.orc_riemann_pool(int(eos_kind), _dp(UL), _dp(UR), ax.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return UL, UR, ax


def fingerprint(F, smax):
    """The order-dependent FNV-1a hash of the bits of every flux and wave speed (cpp/apps/bench_riemann.cpp:86-90)."""
    h = 1469598103934665603
    Fb = np.ascontiguousarray(F, dtype=np.float64).view(np.uint64)
    Sb = np.ascontiguousarray(smax, dtype=np.float64).view(np.uint64)
    mask = (1 << 64) - 1
    for k in range(Fb.shape[0]):
        for q in range(5):
            h = ((h ^ int(Fb[k, q])) * 1099511628211) & mask
        h = ((h ^ int(Sb[k])) * 1099511628211) & mask
    return h


def enstrophy(U, shape, lengths, periodic):
    """1/2 the volume average of |curl u|^2, u = m / rho, with central differences over 2h: the definition of the
    reference's validation scripts (fd_enstrophy, cases/validation/benchmarks/spectra_application.py:61-67: np.roll on a
    periodic box), one-sided over h at the two ends of an axis that is not periodic (as fvg_monitor). shape = (nx, ny, nz),
    lengths = (Lx, Ly, Lz), periodic = three booleans; a mesh with nz = 1 has w_z only."""
    nx, ny, nz = shape
    rho = U[:, 0].reshape(nz, ny, nx)
    vel = [U[:, q].reshape(nz, ny, nx) / rho for q in (1, 2, 4)]
    hs = [lengths[0] / nx, lengths[1] / ny, lengths[2] / nz]

    def d(f, axis):   # axis 0 = x, 1 = y, 2 = z (numpy axes 2, 1, 0)
        ax, h = 2 - axis, hs[axis]
        if periodic[axis]:
            return (np.roll(f, -1, ax) - np.roll(f, 1, ax)) / (2 * h)
        n = f.shape[ax]
        if n == 1:
            return np.zeros_like(f)
        hi = np.take(f, np.minimum(np.arange(n) + 1, n - 1), axis=ax)
        lo = np.take(f, np.maximum(np.arange(n) - 1, 0), axis=ax)
        span = np.full(n, 2.0)
        span[0] -= 1.0
        span[-1] -= 1.0
        sh = [1, 1, 1]
        sh[ax] = n
        return (hi - lo) / (span.reshape(sh) * h)

    u, v, w = vel
    wz = d(v, 0) - d(u, 1)
    if nz == 1:
        return 0.5 * float(np.mean(wz * wz))
    wx = d(w, 1) - d(v, 2)
    wy = d(u, 2) - d(w, 0)
    return 0.5 * float(np.mean(wx * wx + wy * wy + wz * wz))


def ref_available():
    return os.path.exists(REF_SO)


class Reference:
    """The reference solver compiled from its own sources (oracle/_ref/libfenice_ref.so)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_SO):
                raise RuntimeError(f"{REF_SO} is not built (make -C oracle/ref)")
            lib = ctypes.CDLL(REF_SO)
            P = ctypes.POINTER
            lib.ref_error.restype = ctypes.c_char_p
            lib.ref_create.argtypes = [ctypes.c_char_p]
            lib.ref_create.restype = ctypes.c_void_p
            lib.ref_destroy.argtypes = [ctypes.c_void_p]
            lib.ref_dims.argtypes = [ctypes.c_void_p, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]
            lib.ref_time.argtypes = [ctypes.c_void_p]
            lib.ref_time.restype = ctypes.c_double
            lib.ref_dt_length.argtypes = [ctypes.c_void_p]
            lib.ref_dt_length.restype = ctypes.c_double
            lib.ref_lagged_speed.argtypes = [ctypes.c_void_p]
            lib.ref_lagged_speed.restype = ctypes.c_double
            lib.ref_get_state.argtypes = [ctypes.c_void_p, P(ctypes.c_double)]
            lib.ref_set_state.argtypes = [ctypes.c_void_p, P(ctypes.c_double), ctypes.c_int]
            lib.ref_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double]
            lib.ref_residual.argtypes = [ctypes.c_void_p, P(ctypes.c_double), P(ctypes.c_double), ctypes.c_double, ctypes.c_double,
                                         P(ctypes.c_double)]
            lib.ref_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, P(ctypes.c_double), P(ctypes.c_double)]
            lib.ref_solid_mask.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
            lib.ref_ibm_loads.argtypes = [ctypes.c_void_p, P(ctypes.c_double)]
            lib.ref_volume_averages.argtypes = [ctypes.c_void_p, P(ctypes.c_double)]
            lib.ref_cells_create.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.ref_cells_create.restype = ctypes.c_void_p
            lib.ref_cells_destroy.argtypes = [ctypes.c_void_p]
            lib.ref_cells_count.argtypes = [ctypes.c_void_p, P(ctypes.c_int), P(ctypes.c_int)]
            lib.ref_cells_leaves.argtypes = [ctypes.c_void_p] + [P(ctypes.c_int)] * 4
            lib.ref_cells_set_state.argtypes = [ctypes.c_void_p, P(ctypes.c_double)]
            lib.ref_cells_get_state.argtypes = [ctypes.c_void_p, P(ctypes.c_double)]
            lib.ref_cells_residual.argtypes = [ctypes.c_void_p, P(ctypes.c_double), P(ctypes.c_double)]
            lib.ref_cells_steps.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int, P(ctypes.c_double)]
            cls._lib = lib
        return cls._lib

    def __init__(self, params, initial_profile=None, initial_state=None):
        lib = self.lib()
        lines = [f"{k}={v}" for k, v in params.items()]
        if initial_profile:
            lines.append(f"initial_profile={initial_profile}")
        if initial_state is not None:
            lines.append("initial_state=" + ",".join(repr(float(v)) for v in initial_state))
        with quiet_stdout():
            h = lib.ref_create("\n".join(lines).encode())
        if not h:
            raise RuntimeError("reference setup failed: " + lib.ref_error().decode())
        self.h = h
        nx, ny, nz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib.ref_dims(h, ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(nz))
        self.shape = (nx.value, ny.value, nz.value)
        self.ncells = nx.value * ny.value * nz.value

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().ref_destroy(self.h)
            self.h = None

    @property
    def t(self):
        return self.lib().ref_time(self.h)

    @t.setter
    def t(self, value):
        self.lib().ref_set_time(self.h, float(value))

    def dt_length(self):
        return self.lib().ref_dt_length(self.h)

    def lagged_speed(self):
        return self.lib().ref_lagged_speed(self.h)

    def state(self):
        U = np.zeros((self.ncells, 5))
        self.lib().ref_get_state(self.h, _dp(U))
        return U

    def set_state(self, U, force_ibm=False):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (self.ncells, 5)
        self.lib().ref_set_state(self.h, _dp(U), 1 if force_ibm else 0)

    def residual(self, U, stage_time=0.0, predictor_half_dt=0.0):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.zeros_like(U)
        s = ctypes.c_double(0.0)
        rc = self.lib().ref_residual(self.h, _dp(U), _dp(R), float(stage_time), float(predictor_half_dt), ctypes.byref(s))
        if rc:
            raise RuntimeError("reference residual failed: " + self.lib().ref_error().decode())
        return R, s.value

    def steps(self, n, t_end):
        dts = np.zeros(n)
        sms = np.zeros(n)
        k = self.lib().ref_steps(self.h, int(n), float(t_end), _dp(dts), _dp(sms))
        if k < 0:
            raise RuntimeError("reference steps failed: " + self.lib().ref_error().decode())
        return dts[:k], sms[:k]

    def solid_mask(self):
        m = ctypes.create_string_buffer(self.ncells)
        n = self.lib().ref_solid_mask(self.h, m)
        if n < 0:
            return None
        return np.frombuffer(m.raw, dtype=np.int8).copy()

    def volume_averages(self):
        """The monitor's {mass, kinetic energy, total energy} of the current state (Simulation::volume_averages)."""
        v = (ctypes.c_double * 3)()
        self.lib().ref_volume_averages(self.h, v)
        return list(v)

    def ibm_loads(self):
        """{Fx, Fy, Mz} of the immersed body from a residual of the current state (Simulation::ibm_loads)."""
        v = (ctypes.c_double * 3)()
        if self.lib().ref_ibm_loads(self.h, v) != 0:
            raise RuntimeError("reference ibm_loads failed: " + self.lib().ref_error().decode())
        return list(v)


class ReferenceCells:
    """The reference's cell engine of an adaptive mesh on a Reference run's objects (ref_cells_* of the harness): the
    CellMesh of the run's base mesh (levels 0 .. max_level, every leaf of level 0 as built), its CellFluxEngine and a
    CellAdvance with the run's time scheme, as the reference's level-0 tests make them. Keep the Reference alive."""

    def __init__(self, ref, max_level=0):
        lib = Reference.lib()
        self.ref = ref
        self.h = lib.ref_cells_create(ref.h, int(max_level))
        if not self.h:
            raise RuntimeError("reference cell engine failed: " + lib.ref_error().decode())
        n, nf = ctypes.c_int(), ctypes.c_int()
        lib.ref_cells_count(self.h, ctypes.byref(n), ctypes.byref(nf))
        self.nleaf, self.nface = n.value, nf.value
        arrs = [np.zeros(self.nleaf, dtype=np.int32) for _ in range(4)]
        lib.ref_cells_leaves(self.h, *[a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) for a in arrs])
        self.level, self.ci, self.cj, self.ck = arrs

    def __del__(self):
        if getattr(self, "h", None):
            Reference.lib().ref_cells_destroy(self.h)
            self.h = None

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (self.nleaf, 5)
        Reference.lib().ref_cells_set_state(self.h, _dp(U))

    def state(self):
        U = np.zeros((self.nleaf, 5))
        Reference.lib().ref_cells_get_state(self.h, _dp(U))
        return U

    def residual(self):
        """(R, largest face speed) of the state held (CellFluxEngine::residual)."""
        R = np.zeros((self.nleaf, 5))
        s = ctypes.c_double(0.0)
        if Reference.lib().ref_cells_residual(self.h, _dp(R), ctypes.byref(s)):
            raise RuntimeError("reference cell residual failed: " + Reference.lib().ref_error().decode())
        return R, s.value

    def steps(self, dt, n, t0=0.0):
        """n CellAdvance::step(dt, t0 + k dt); the speed each returned."""
        s = np.zeros(n)
        if Reference.lib().ref_cells_steps(self.h, float(dt), float(t0), int(n), _dp(s)):
            raise RuntimeError("reference cell steps failed: " + Reference.lib().ref_error().decode())
        return s

