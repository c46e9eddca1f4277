"""Python host binding of the C ABI (include/fenice_gpu.h, fenice_b200/libfenice_gpu.so).

``Run`` mirrors the reference's hot-path interface: ``residual(U)`` is Simulation::residual (returns R and the wave
speed, cpp/src/Simulation.cpp:1351-1354), ``step(t_end)`` one pass of the serial time loop (TimeScheme::step +
check_progress + t += dt, cpp/src/SimulationRun.cpp:441-464) returning the reference's StepResult {dt, s_max}, and
``run(t_end, max_steps)`` the loop itself. States are (ncells, 5) float64 arrays in the reference's layout. Failures
raise: ValueError for a configuration the reference rejects or this build does not support, RuntimeError for a
diverged run (the reference's std::runtime_error of check_progress) or a CUDA failure.

There is no CPU fallback: without the CUDA library or a device every call raises.
"""
import ctypes
import os
from collections import namedtuple

import numpy as np

from . import params as P

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfenice_gpu.so")

FVG_OK, FVG_ERR_CONFIG, FVG_ERR_ARGUMENT, FVG_ERR_CUDA, FVG_ERR_DIVERGED, FVG_ERR_STATE, FVG_ERR_BOUNDARY = range(7)

StepResult = namedtuple("StepResult", ["dt", "s_max"])

# every entry point of include/fenice_gpu.h
EXPORTS = ["fvg_abi_version", "fvg_create", "fvg_destroy", "fvg_last_error", "fvg_create_error", "fvg_upload_state",
           "fvg_download_state", "fvg_residual", "fvg_step", "fvg_run_until", "fvg_step_host", "fvg_get_time", "fvg_set_time", "fvg_set_stage_time",
           "fvg_get_lagged_speed", "fvg_set_lagged_speed", "fvg_dt_length", "fvg_device_state", "fvg_stream",
           "fvg_synchronize", "fvg_face_flux_batch", "fvg_set_timing", "fvg_get_timing",
           "fvg_residual_noalloc",
           "fvg_batch_create", "fvg_batch_destroy", "fvg_batch_last_error", "fvg_batch_cells", "fvg_batch_upload",
           "fvg_batch_download", "fvg_batch_run", "fvg_batch_problem", "fvg_batch_autotune", "fvg_batch_set_schedule",
           "fvg_batch_get_schedule", "fvg_batch_stream", "fvg_batch_set_timing", "fvg_batch_get_timing",
           "fvg_sensor_sizes", "fvg_sensor_extract", "fvg_sensor_grad", "fvg_sensor_adam", "fvg_sensor_pack", "fvg_sensor_infer",
           "fvg_set_sensor", "fvg_get_sensor_counts", "fvg_get_sensor_gate", "fvg_ibm_loads", "fvg_monitor", "fvg_get_body_state", "fvg_set_body_state",
           "fvg_create_part", "fvg_part_info", "fvg_part_buffers", "fvg_part_begin", "fvg_part_phase", "fvg_part_status",
           "fvg_expr_eval",
           "fvg_cells_create", "fvg_cells_destroy", "fvg_cells_last_error", "fvg_cells_info", "fvg_cells_upload_state",
           "fvg_cells_download_state", "fvg_cells_residual", "fvg_cells_step", "fvg_cells_advance", "fvg_cells_stream"]

_lib = None
ABI_VERSION = 9   # FVG_ABI_VERSION of include/fenice_gpu.h


def load_library(path=LIB_PATH):
    """The CUDA library, loaded once (ctypes); raises if it was not built (python -m fenice_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m fenice_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(path)
    c_p = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    lib.fvg_abi_version.restype = ctypes.c_int
    if lib.fvg_abi_version() != ABI_VERSION:   # fvg_config's layout is the one params.FvgConfig mirrors
        raise RuntimeError(f"{path} has ABI version {lib.fvg_abi_version()}, this package needs {ABI_VERSION}: rebuild it")
    lib.fvg_create.argtypes = [ctypes.POINTER(P.FvgConfig), ctypes.POINTER(c_p)]
    lib.fvg_destroy.argtypes = [c_p]
    lib.fvg_last_error.argtypes = [c_p]
    lib.fvg_last_error.restype = ctypes.c_char_p
    lib.fvg_create_error.restype = ctypes.c_char_p
    lib.fvg_upload_state.argtypes = [c_p, dp, ctypes.c_size_t]
    lib.fvg_download_state.argtypes = [c_p, dp, ctypes.c_size_t]
    lib.fvg_residual.argtypes = [c_p, ctypes.c_double, dp, ctypes.c_size_t, dp]
    lib.fvg_step.argtypes = [c_p, ctypes.c_double, dp, dp]
    lib.fvg_step_host.argtypes = [c_p, dp, dp, ctypes.c_size_t, ctypes.c_double, dp, dp]
    lib.fvg_run_until.argtypes = [c_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.fvg_get_time.argtypes = [c_p, dp]
    lib.fvg_set_time.argtypes = [c_p, ctypes.c_double]
    lib.fvg_set_stage_time.argtypes = [c_p, ctypes.c_double]
    lib.fvg_get_lagged_speed.argtypes = [c_p, dp]
    lib.fvg_set_lagged_speed.argtypes = [c_p, ctypes.c_double]
    lib.fvg_dt_length.argtypes = [c_p, dp]
    lib.fvg_device_state.argtypes = [c_p, ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
    lib.fvg_stream.argtypes = [c_p, ctypes.POINTER(c_p)]
    lib.fvg_synchronize.argtypes = [c_p]
    lib.fvg_face_flux_batch.argtypes = [c_p, dp, dp, ctypes.POINTER(ctypes.c_int), ctypes.c_size_t, dp, dp]
    lib.fvg_residual_noalloc.argtypes = [ctypes.POINTER(P.FvgConfig), c_p, ctypes.c_longlong, c_p, dp, c_p]
    lib.fvg_set_timing.argtypes = [c_p, ctypes.c_int]
    ll = ctypes.POINTER(ctypes.c_longlong)
    lib.fvg_get_timing.argtypes = [c_p, dp, ll, dp, ll]
    ip = ctypes.POINTER(ctypes.c_int)
    lib.fvg_batch_create.argtypes = [ctypes.POINTER(P.FvgConfig), ctypes.c_int, ctypes.POINTER(c_p)]
    lib.fvg_batch_destroy.argtypes = [c_p]
    lib.fvg_batch_last_error.argtypes = [c_p]
    lib.fvg_batch_last_error.restype = ctypes.c_char_p
    lib.fvg_batch_cells.argtypes = [c_p, ll]
    lib.fvg_batch_upload.argtypes = [c_p, dp, ctypes.c_size_t]
    lib.fvg_batch_download.argtypes = [c_p, dp, ctypes.c_size_t]
    lib.fvg_batch_run.argtypes = [c_p, ctypes.c_double, ctypes.c_int, ll]
    lib.fvg_batch_problem.argtypes = [c_p, ctypes.c_int, dp, ip, ip]
    lib.fvg_batch_autotune.argtypes = [c_p, ip, ip, dp]
    lib.fvg_batch_set_schedule.argtypes = [c_p, ctypes.c_int, ctypes.c_int]
    lib.fvg_batch_get_schedule.argtypes = [c_p, ip, ip, ip, ip]
    lib.fvg_batch_stream.argtypes = [c_p, ctypes.POINTER(c_p)]
    lib.fvg_batch_set_timing.argtypes = [c_p, ctypes.c_int]
    lib.fvg_batch_get_timing.argtypes = [c_p, dp, ll]
    lib.fvg_sensor_sizes.argtypes = [ip, ip, ip]
    lib.fvg_sensor_extract.argtypes = [c_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_float, c_p, c_p, c_p, ctypes.c_longlong, c_p]
    lib.fvg_sensor_grad.argtypes = [c_p, c_p, c_p, ctypes.c_longlong, ctypes.c_float, c_p, c_p, c_p]
    lib.fvg_sensor_adam.argtypes = [c_p, c_p, c_p, c_p, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, c_p, c_p]
    lib.fvg_sensor_pack.argtypes = [c_p, c_p, c_p]
    lib.fvg_sensor_infer.argtypes = [c_p, c_p, ctypes.c_longlong, c_p, c_p]
    lib.fvg_set_sensor.argtypes = [c_p, c_p, ctypes.c_float, ctypes.c_int, ctypes.c_int]
    lib.fvg_get_sensor_counts.argtypes = [c_p, ll, ll, ctypes.c_int]
    lib.fvg_get_sensor_gate.argtypes = [c_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.fvg_ibm_loads.argtypes = [c_p, dp]
    lib.fvg_monitor.argtypes = [c_p, ctypes.c_int, dp]
    lib.fvg_get_body_state.argtypes = [c_p, dp, ctypes.POINTER(ctypes.c_int)]
    lib.fvg_set_body_state.argtypes = [c_p, dp, ctypes.c_int]
    ip = ctypes.POINTER(ctypes.c_int)
    dpp = ctypes.POINTER(dp)
    lib.fvg_create_part.argtypes = [ctypes.POINTER(P.FvgConfig), ctypes.c_int, ctypes.c_int, ctypes.POINTER(c_p)]
    lib.fvg_part_info.argtypes = [c_p, ip, ip, ip, ip, ip, ip]
    lib.fvg_part_buffers.argtypes = [c_p, dpp, dpp, dpp, dpp, ll, dpp]
    lib.fvg_part_begin.argtypes = [c_p, ctypes.c_double, ctypes.c_int]
    lib.fvg_part_phase.argtypes = [c_p, ctypes.c_int, ip, ip]
    lib.fvg_part_status.argtypes = [c_p, ip, ip, dp, dp, dp]
    lib.fvg_expr_eval.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), dp, ctypes.c_int, dp, dp, dp, ctypes.c_double, ctypes.c_size_t, dp,
                                  ctypes.c_char_p, ctypes.c_size_t]
    lib.fvg_cells_create.argtypes = [ctypes.POINTER(P.FvgConfig), ctypes.c_int, ip, ip, ip, ip, ctypes.POINTER(c_p)]
    lib.fvg_cells_destroy.argtypes = [c_p]
    lib.fvg_cells_last_error.argtypes = [c_p]
    lib.fvg_cells_last_error.restype = ctypes.c_char_p
    lib.fvg_cells_info.argtypes = [c_p, ll, ll]
    lib.fvg_cells_upload_state.argtypes = [c_p, dp, ctypes.c_size_t]
    lib.fvg_cells_download_state.argtypes = [c_p, dp, ctypes.c_size_t]
    lib.fvg_cells_residual.argtypes = [c_p, dp, ctypes.c_size_t, dp]
    lib.fvg_cells_step.argtypes = [c_p, ctypes.c_double, ctypes.c_double, dp]
    lib.fvg_cells_advance.argtypes = [c_p, ctypes.c_double, ctypes.c_int, dp]
    lib.fvg_cells_stream.argtypes = [c_p, ctypes.POINTER(c_p)]
    _lib = lib
    return lib


def eval_expression(src, names, x, y, z, t=0.0):
    """A case-file expression evaluated on the host by the library's compiler (fvg_expr_eval: the reference's grammar
    and the C library's functions) at the points (x, y, z) and time t. `names`: a dict or (name, value) pairs bound
    after x, y, z, t (later ones replace earlier ones). ValueError for an expression the grammar refuses."""
    lib = load_library()
    pairs = list(names.items()) if isinstance(names, dict) else list(names)
    n = len(x)
    arrs = [np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (n,))) for a in (x, y, z)]
    out = np.empty(n)
    cn = (ctypes.c_char_p * max(1, len(pairs)))(*[k.encode() for k, _ in pairs])
    cv = np.array([float(v) for _, v in pairs] or [0.0])
    err = ctypes.create_string_buffer(512)
    rc = lib.fvg_expr_eval(str(src).encode(), cn, _dp(cv), len(pairs), _dp(arrs[0]), _dp(arrs[1]), _dp(arrs[2]), float(t), n, _dp(out), err, 512)
    if rc != 0:
        raise ValueError(err.value.decode())
    return out


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Run:
    """A run of the finite-volume path on one GPU."""

    def __init__(self, params, U=None, precision=0, device=0, part=None):
        """part = (nparts, index): one part of the slab decomposition of the mesh (fvg_create_part; see
        fenice_b200.slabs), whose state is its own planes."""
        self.lib = load_library()
        self.params = P.resolve(params)
        self.cfg = P.to_config(self.params, precision=precision, device=device)
        h = ctypes.c_void_p()
        if part is None:
            rc = self.lib.fvg_create(ctypes.byref(self.cfg), ctypes.byref(h))
        else:
            rc = self.lib.fvg_create_part(ctypes.byref(self.cfg), int(part[0]), int(part[1]), ctypes.byref(h))
        if rc != FVG_OK:
            msg = self.lib.fvg_create_error().decode()
            raise (ValueError if rc in (FVG_ERR_CONFIG, FVG_ERR_ARGUMENT) else RuntimeError)(f"fvg_create: {msg}")
        self.h = h
        self.shape = (self.cfg.nx, self.cfg.ny, self.cfg.nz)
        if part is not None:
            ax, first, count = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            self.lib.fvg_part_info(h, ctypes.byref(ax), ctypes.byref(first), ctypes.byref(count), None, None, None)
            shape = list(self.shape)
            shape[ax.value] = count.value
            self.shape = tuple(shape)
        self.ncells = self.shape[0] * self.shape[1] * self.shape[2]
        self.stages = P.STAGES[self.cfg.time_scheme]
        if U is not None:
            self.set_state(U)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fvg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc, what):
        if rc == FVG_OK:
            return
        msg = self.lib.fvg_last_error(self.h).decode()
        if rc in (FVG_ERR_CONFIG, FVG_ERR_ARGUMENT, FVG_ERR_STATE):
            raise ValueError(f"{what}: {msg}")
        raise RuntimeError(f"{what}: {msg}")

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (self.ncells, 5):
            raise ValueError(f"state must be ({self.ncells}, 5), got {U.shape}")
        self._check(self.lib.fvg_upload_state(self.h, _dp(U), self.ncells), "upload")

    def state(self, out=None):
        """The state (a new array, or `out`: a C-contiguous float64 (ncells, 5) array, e.g. a view of pinned memory, which
        the device then writes directly)."""
        U = np.empty((self.ncells, 5)) if out is None else out
        if U.shape != (self.ncells, 5) or U.dtype != np.float64 or not U.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (ncells, 5)")
        self._check(self.lib.fvg_download_state(self.h, _dp(U), self.ncells), "download")
        return U

    def residual(self, U=None, predictor_half_dt=0.0, want_R=True):
        """R and the wave speed of U (default: the run's state), as Simulation::residual."""
        if U is not None:
            self.set_state(U)
        R = np.empty((self.ncells, 5)) if want_R else None
        s = ctypes.c_double()
        self._check(self.lib.fvg_residual(self.h, float(predictor_half_dt), _dp(R) if want_R else None, self.ncells if want_R else 0,
                                          ctypes.byref(s)), "residual")
        return R, s.value

    def set_stage_time(self, t=float("nan")):
        """The time at which the next residual() evaluates time-dependent source terms and boundary values
        (TimeScheme::stage_time); NaN: the run's time (plus predictor_half_dt for a MUSCL-Hancock residual)."""
        self._check(self.lib.fvg_set_stage_time(self.h, float(t)), "stage time")

    def step(self, t_end):
        dt, s = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.fvg_step(self.h, float(t_end), ctypes.byref(dt), ctypes.byref(s)), "step")
        return StepResult(dt.value, s.value)

    def step_host(self, U, t_end, out=None):
        """One step of a state held in host memory (TimeScheme::step(Field& U) with the caller's U): U is uploaded, stepped
        toward t_end and the new state written to `out` (default: U itself, in place). U and out are C-contiguous float64
        (ncells, 5) arrays; in pinned memory (e.g. views of torch pin_memory tensors) the copies overlap the computation.
        The result is the bits of set_state + step + state."""
        out = U if out is None else out
        for a, name in ((U, "U"), (out, "out")):
            if not isinstance(a, np.ndarray) or a.shape != (self.ncells, 5) or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError(f"{name} must be a C-contiguous float64 array of shape ({self.ncells}, 5)")
        if not out.flags.writeable:
            raise ValueError("out must be writeable")
        dt, s = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.fvg_step_host(self.h, _dp(U), _dp(out), self.ncells, float(t_end), ctypes.byref(dt), ctypes.byref(s)), "step_host")
        return StepResult(dt.value, s.value)

    def run(self, t_end, max_steps=0):
        """Steps until t >= t_end or max_steps steps (graph-captured); returns the number of steps."""
        n = ctypes.c_int()
        self._check(self.lib.fvg_run_until(self.h, float(t_end), int(max_steps), ctypes.byref(n)), "run")
        return n.value

    @property
    def t(self):
        v = ctypes.c_double()
        self._check(self.lib.fvg_get_time(self.h, ctypes.byref(v)), "time")
        return v.value

    @t.setter
    def t(self, value):
        self._check(self.lib.fvg_set_time(self.h, float(value)), "time")

    @property
    def lagged_speed(self):
        v = ctypes.c_double()
        self._check(self.lib.fvg_get_lagged_speed(self.h, ctypes.byref(v)), "lagged speed")
        return v.value

    @lagged_speed.setter
    def lagged_speed(self, value):
        self._check(self.lib.fvg_set_lagged_speed(self.h, float(value)), "lagged speed")

    def dt_length(self):
        v = ctypes.c_double()
        self._check(self.lib.fvg_dt_length(self.h, ctypes.byref(v)), "dt_length")
        return v.value

    def device_state(self):
        """(device pointer, plane stride in doubles, nvar) of the state planes."""
        ptr = ctypes.POINTER(ctypes.c_double)()
        plane, nvar = ctypes.c_longlong(), ctypes.c_int()
        self._check(self.lib.fvg_device_state(self.h, ctypes.byref(ptr), ctypes.byref(plane), ctypes.byref(nvar)), "device_state")
        return ctypes.cast(ptr, ctypes.c_void_p).value, plane.value, nvar.value

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self.lib.fvg_stream(self.h, ctypes.byref(s)), "stream")
        return s.value

    def synchronize(self):
        self._check(self.lib.fvg_synchronize(self.h), "synchronize")

    def set_timing(self, on=True):
        self._check(self.lib.fvg_set_timing(self.h, 1 if on else 0), "set_timing")

    def timing(self):
        """{stage_ms, stage_launches, viscous_ms, viscous_launches} summed since set_timing(True)."""
        a, b, c, d = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double(), ctypes.c_longlong()
        self._check(self.lib.fvg_get_timing(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d)), "get_timing")
        return {"stage_ms": a.value, "stage_launches": b.value, "viscous_ms": c.value, "viscous_launches": d.value}

    def ibm_loads(self):
        """{Fx, Fy, Mz, Cd, Cl, Cm} of the immersed body from a residual of the current state (Simulation::ibm_loads and
        the monitor's coefficients)."""
        v = (ctypes.c_double * 6)()
        self._check(self.lib.fvg_ibm_loads(self.h, v), "ibm_loads")
        return dict(zip(["Fx", "Fy", "Mz", "Cd", "Cl", "Cm"], list(v)))

    @property
    def body_state(self):
        """The moving body's state in the reference's checkpoint layout (body_pose; fvg_get_body_state), or None without a
        moving body. Assigning restores it (set the time first)."""
        n = ctypes.c_int(0)
        self._check(self.lib.fvg_get_body_state(self.h, None, ctypes.byref(n)), "get_body_state")
        if n.value == 0:
            return None
        v = np.zeros(n.value)
        self._check(self.lib.fvg_get_body_state(self.h, _dp(v), ctypes.byref(n)), "get_body_state")
        return v

    @body_state.setter
    def body_state(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        self._check(self.lib.fvg_set_body_state(self.h, _dp(v), int(v.size)), "set_body_state")

    def monitor(self, order="reference"):
        """{mass, kinetic_energy, total_energy, enstrophy} of the current state (fvg_monitor): the volume averages of the
        reference's monitor file and 1/2 <|curl u|^2>. order "reference": its summation order (its bits; one device
        thread), "fast": a fixed parallel order (within rounding of it)."""
        v = (ctypes.c_double * 4)()
        self._check(self.lib.fvg_monitor(self.h, 0 if order == "reference" else 1, v), "monitor")
        return dict(zip(["mass", "kinetic_energy", "total_energy", "enstrophy"], list(v)))

    def set_sensor(self, sensor, threshold=0.0, every=0, radius=-1):
        """Gate the WENO5-Z reconstructions (mixed precision) with a trained ``fenice_b200.sensor.Sensor`` (None: off),
        refreshed every `every` steps and grown by `radius` cells (defaults: 10 steps, ceil(cfl every) + 1 cells)."""
        ptr = None if sensor is None else sensor.weights_ptr()
        self._check(self.lib.fvg_set_sensor(self.h, ptr, float(threshold), int(every), int(radius)), "set_sensor")

    def sensor_gate(self):
        """The gate of the last refresh: (cell_flags (dim, ncells) uint8: the network's flag of every (cell, axis), 1 = stays
        WENO5-Z; tile_flags (dim, tiles z, tiles y, tiles x) uint8: what the stage kernels read; the tile's cells (x, y, z))."""
        dim = 3 if int(self.params.get("nz", 1)) > 1 else 2
        tile, tiles = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        self._check(self.lib.fvg_get_sensor_gate(self.h, None, None, tile, tiles), "sensor_gate")
        cells = np.empty((dim, self.ncells), dtype=np.uint8)
        tf = np.empty((dim, tiles[2], tiles[1], tiles[0]), dtype=np.uint8)
        self._check(self.lib.fvg_get_sensor_gate(self.h, cells.ctypes.data, tf.ctypes.data, tile, tiles), "sensor_gate")
        return cells, tf, tuple(tile)

    def sensor_counts(self, reset=False):
        """(cell-axis evaluations that went linear, all evaluations) since the last reset."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.fvg_get_sensor_counts(self.h, ctypes.byref(a), ctypes.byref(b), 1 if reset else 0), "sensor_counts")
        return a.value, b.value

    def face_flux_batch(self, UL, UR, axis):
        UL = np.ascontiguousarray(UL, dtype=np.float64)
        UR = np.ascontiguousarray(UR, dtype=np.float64)
        ax = np.ascontiguousarray(axis, dtype=np.int32)
        n = UL.shape[0]
        F = np.empty((n, 5))
        S = np.empty(n)
        self._check(self.lib.fvg_face_flux_batch(self.h, _dp(UL), _dp(UR), ax.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n, _dp(F), _dp(S)),
                    "face_flux_batch")
        return F, S


BatchProblem = namedtuple("BatchProblem", ["t", "steps", "status"])


def batch_cost(params):
    """Relative cost of a problem: cells x steps, with steps proportional to 1 / (cfl L), L = min(dx, dy)."""
    p = P.resolve(params)
    nx, ny = int(p["nx"]), int(p["ny"])
    L = min(float(p["Lx"]) / nx, float(p["Ly"]) / ny)
    return nx * ny / (float(p["cfl"]) * L)


def split_batch(params_list, parts):
    """Problem indices for each of `parts` GPUs: longest-processing-time-first by batch_cost, so the most loaded GPU
    carries as little as the greedy rule gets it (the batch has no exchange between problems)."""
    cost = [batch_cost(p) for p in params_list]
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(cost)), key=lambda k: (-cost[k], k)):
        r = min(range(parts), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += cost[i]
    return [sorted(o) for o in out]


class Batch:
    """Independent 2-D problems of uneven sizes advanced together on one GPU (fvg_batch_*): one persistent launch per
    Runge-Kutta stage for all of them, each problem with its own clock, dt and step count, each getting the bits its
    single ``Run`` gives. ``params_list`` holds one parameter dict per problem (reference keys); the problems share the
    scheme. States are (sum of cells, 5) float64 arrays: problem 0's cells, then problem 1's, ..."""

    def __init__(self, params_list, states=None, precision=0, device=0):
        self.lib = load_library()
        self.params = [P.resolve(p) for p in params_list]
        n = len(self.params)
        cfgs = (P.FvgConfig * n)(*[P.to_config(p, precision=precision, device=device) for p in self.params])
        self.cfgs = cfgs
        h = ctypes.c_void_p()
        rc = self.lib.fvg_batch_create(cfgs, n, ctypes.byref(h))
        if rc != FVG_OK:
            msg = self.lib.fvg_create_error().decode()
            raise (ValueError if rc == FVG_ERR_CONFIG else RuntimeError)(f"fvg_batch_create: {msg}")
        self.h = h
        self.n = n
        self.cells = [c.nx * c.ny for c in cfgs]
        self.offsets = np.concatenate([[0], np.cumsum(self.cells)]).astype(np.int64)
        self.ncells = int(self.offsets[-1])
        self.stages = P.STAGES[cfgs[0].time_scheme]
        if states is not None:
            self.set_state(np.concatenate(states) if isinstance(states, (list, tuple)) else states)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fvg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc, what):
        if rc == FVG_OK:
            return
        msg = self.lib.fvg_batch_last_error(self.h).decode()
        if rc in (FVG_ERR_CONFIG, FVG_ERR_ARGUMENT, FVG_ERR_STATE):
            raise ValueError(f"{what}: {msg}")
        raise RuntimeError(f"{what}: {msg}")

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (self.ncells, 5):
            raise ValueError(f"state must be ({self.ncells}, 5), got {U.shape}")
        self._check(self.lib.fvg_batch_upload(self.h, _dp(U), self.ncells), "upload")

    def state(self, out=None):
        U = np.empty((self.ncells, 5)) if out is None else out
        if U.shape != (self.ncells, 5) or U.dtype != np.float64 or not U.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (ncells, 5)")
        self._check(self.lib.fvg_batch_download(self.h, _dp(U), self.ncells), "download")
        return U

    def split(self, U):
        """The per-problem views of a batch state array."""
        return [U[self.offsets[p]:self.offsets[p + 1]] for p in range(self.n)]

    def run(self, t_end, max_steps=0, check=True):
        """Every problem to t_end (or max_steps steps); returns the cell-stages done. A diverged problem raises
        RuntimeError after the others finished (check=False: no raise; see problem(i).status)."""
        w = ctypes.c_longlong()
        rc = self.lib.fvg_batch_run(self.h, float(t_end), int(max_steps), ctypes.byref(w))
        if check or rc != FVG_ERR_DIVERGED:
            self._check(rc, "run")
        return w.value

    def problem(self, i):
        t, s, st = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.fvg_batch_problem(self.h, int(i), ctypes.byref(t), ctypes.byref(s), ctypes.byref(st)), "problem")
        return BatchProblem(t.value, s.value, st.value)

    def autotune(self):
        """Picks the tile shape and persistent grid (fvg_batch_autotune); returns (shape, ctas_per_sm, stage_ms)."""
        s, c, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.fvg_batch_autotune(self.h, ctypes.byref(s), ctypes.byref(c), ctypes.byref(ms)), "autotune")
        return s.value, c.value, ms.value

    def set_schedule(self, shape, ctas_per_sm=0):
        self._check(self.lib.fvg_batch_set_schedule(self.h, int(shape), int(ctas_per_sm)), "set_schedule")

    def schedule(self):
        """{shape, tile_x, tile_y, grid} (shape -1: not chosen yet)"""
        v = [ctypes.c_int() for _ in range(4)]
        self._check(self.lib.fvg_batch_get_schedule(self.h, *[ctypes.byref(x) for x in v]), "get_schedule")
        return dict(zip(["shape", "tile_x", "tile_y", "grid"], [x.value for x in v]))

    def stream(self):
        s = ctypes.c_void_p()
        self._check(self.lib.fvg_batch_stream(self.h, ctypes.byref(s)), "stream")
        return s.value

    def set_timing(self, on=True):
        self._check(self.lib.fvg_batch_set_timing(self.h, 1 if on else 0), "set_timing")

    def timing(self):
        a, b = ctypes.c_double(), ctypes.c_longlong()
        self._check(self.lib.fvg_batch_get_timing(self.h, ctypes.byref(a), ctypes.byref(b)), "get_timing")
        return {"stage_ms": a.value, "stage_launches": b.value}
