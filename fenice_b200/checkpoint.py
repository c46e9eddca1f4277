"""Checkpoints and final-state dumps in the reference's file format, so a run on the device resumes from a checkpoint the
reference wrote and the reference resumes from one written here.

Checkpoint (Simulation::checkpoint_header / save_checkpoint / load_checkpoint, cpp/src/SimulationRestart.cpp:61-85,
162-189, 254-360, format_version 1): an uncompressed .npz (the reference's reader refuses np.savez_compressed) with
  format_version  int64 scalar, 1 (a file with a higher number is refused)
  t, step         float64 / int64 scalars
  nx, ny, nz      int64 scalars; Lx, Ly, Lz float64 scalars
  S               float64 scalar, the MUSCL-Hancock lagged wave speed (only when the scheme has one > 0)
  collection_time, collection_file   float64 (n,) and <U (n,): the output index of the run (empty here)
  U               float64 (ncells, 4) on a 2-D mesh (rho w left out), (ncells, 5) in 3-D, the reference's cell order
  body_pose       float64 (10, 13, 14 or 21,): a moving immersed body's pose and state (Simulation::body_checkpoint,
                  SimulationRestart.cpp:87-97; only for a run with a moving body, which refuses a file without it, :103)
written to <path>_tmp.npz and renamed over the file, as the reference does. An adaptive (AMR) checkpoint (leaf_level ...)
is refused.

Final-state dump (Simulation::dump_final_state, SimulationRestart.cpp:449-476; the `dump_state` option): t, step, U.
"""
import os

import numpy as np

FORMAT_VERSION = 1


def _u_columns(run):
    return 5 if run.shape[2] > 1 else 4


def _write(path, arrays):
    tmp = path[:-4] + "_tmp.npz" if path.endswith(".npz") else path + "_tmp.npz"
    with open(tmp, "wb") as f:
        np.savez(f, **arrays)
    os.replace(tmp, path)


def checkpoint_arrays(U, t, step, params, lagged_speed=0.0, collection=(), body_pose=None):
    """The arrays of a checkpoint (checkpoint_header + U): U of 5 columns per cell (rho w dropped on a 2-D mesh), the
    resolved parameters of the run (nx .. Lz), the MUSCL-Hancock lagged speed (written when > 0), the output index, the
    moving body's body_pose (when given)."""
    nx, ny, nz = int(params["nx"]), int(params["ny"]), int(params.get("nz", 1))
    times = np.array([float(tc) for tc, _ in collection], dtype=np.float64)
    files = [str(f) for _, f in collection]
    a = {}
    if lagged_speed > 0.0:
        a["S"] = np.array(float(lagged_speed), dtype=np.float64)
    a.update(format_version=np.array(FORMAT_VERSION, dtype=np.int64), t=np.array(float(t), dtype=np.float64), step=np.array(int(step), dtype=np.int64),
             nx=np.array(nx, dtype=np.int64), ny=np.array(ny, dtype=np.int64), Lx=np.array(float(params["Lx"]), dtype=np.float64),
             Ly=np.array(float(params["Ly"]), dtype=np.float64), nz=np.array(nz, dtype=np.int64), Lz=np.array(float(params["Lz"]), dtype=np.float64),
             collection_time=times, collection_file=np.array(files, dtype=f"<U{max([1] + [len(f) for f in files])}"),
             U=np.ascontiguousarray(np.asarray(U, dtype=np.float64)[:, :5 if nz > 1 else 4]))
    if body_pose is not None:
        a["body_pose"] = np.ascontiguousarray(np.asarray(body_pose, dtype=np.float64).ravel())
    return a


def write_checkpoint(path, arrays):
    """Writes checkpoint arrays as the reference does: an uncompressed .npz, through <path>_tmp.npz renamed over it."""
    _write(path, arrays)


def save_checkpoint(path, run, step, collection=()):
    """Writes the run's state, time and step (and, for MUSCL-Hancock, its lagged speed; for a moving body, its pose) as
    the reference's checkpoint."""
    s = run.lagged_speed if run.cfg.time_scheme == 3 else 0.0
    _write(path, checkpoint_arrays(run.state(), run.t, step, run.params, s, collection, run.body_state))


def read_checkpoint(path):
    """The arrays of a reference checkpoint (a dict), after the reference's checks: known format, a uniform mesh."""
    with np.load(path, allow_pickle=False) as z:
        a = {k: z[k] for k in z.files}
    if "format_version" in a and int(a["format_version"]) > FORMAT_VERSION:
        raise ValueError(f"The checkpoint {path} has format_version {int(a['format_version'])}, newer than this reader ({FORMAT_VERSION})")
    if "leaf_level" in a:
        raise ValueError(f"The checkpoint {path} is from an adaptive (AMR) run; the device path runs uniform meshes")
    U = a.get("U")
    if U is None or U.ndim != 2 or U.shape[1] not in (4, 5):
        raise ValueError(f"The checkpoint {path} has no (n, 4) or (n, 5) state array U")
    return a


def load_checkpoint(path, run):
    """Resumes `run` from a checkpoint (the reference's or save_checkpoint's): its state, time and, when present, the
    MUSCL-Hancock lagged speed (a checkpoint of another scheme has none: the first step seeds it). Returns the step."""
    a = read_checkpoint(path)
    for key, n in (("nx", run.params["nx"]), ("ny", run.params["ny"]), ("nz", run.params["nz"])):
        if key in a and int(a[key]) != int(n):
            raise ValueError(f"The checkpoint {path} is of a {int(a['nx'])} x {int(a['ny'])} x {int(a['nz'])} mesh, the run's is "
                             f"{run.params['nx']} x {run.params['ny']} x {run.params['nz']}")
    # the domain's size as well, 1e-10 apart at most (the reference's test for the base mesh of an adaptive file,
    # SimulationRestart.cpp:283-287; a uniform file of another size would resume with another spacing)
    for key in ("Lx", "Ly", "Lz"):
        if key in a and abs(float(a[key]) - float(run.params[key])) > 1e-10:
            raise ValueError(f"The checkpoint {path} is of a domain with {key} = {float(a[key])!r}, the run's is {float(run.params[key])!r}")
    U = np.asarray(a["U"], dtype=np.float64)
    if U.shape[0] != run.ncells:
        raise ValueError(f"The checkpoint {path} holds {U.shape[0]} cells, the run {run.ncells}")
    full = np.zeros((run.ncells, 5))
    full[:, :U.shape[1]] = U
    moving = run.body_state is not None
    if moving and "body_pose" not in a:   # SimulationRestart.cpp:103
        raise ValueError(f"The checkpoint {path} has no pose of the moving body: it is from a static run")
    run.set_state(full)
    run.t = float(a["t"])
    if run.cfg.time_scheme == 3:
        run.lagged_speed = float(a["S"]) if "S" in a else 0.0
    if moving:
        run.body_state = np.asarray(a["body_pose"], dtype=np.float64)
    return int(a["step"])


def dump_state(path, run, step):
    """The reference's final-state dump (dump_state): t, step, U."""
    U = run.state()
    _write(path, {"t": np.array(run.t, dtype=np.float64), "step": np.array(int(step), dtype=np.int64), "U": np.ascontiguousarray(U[:, :_u_columns(run)])})


def read_dump(path):
    """(U with 5 columns, t, step) of a dump_state file."""
    with np.load(path, allow_pickle=False) as z:
        U = np.asarray(z["U"], dtype=np.float64)
        full = np.zeros((U.shape[0], 5))
        full[:, :U.shape[1]] = U
        return full, float(z["t"]), int(z["step"])
