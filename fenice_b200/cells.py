"""The cell engine of an adaptive mesh on the GPU, for meshes whose leaves are all of level 0 (fvg_cells_*).

The reference's AMR engine keeps a CellMesh (cpp/include/fv/CellMesh.hpp: leaves sorted by level and Morton key, their
faces and side lists), computes its residual with a CellFluxEngine (cpp/include/fv/CellFlux.hpp:92-270; one flux per
face from stencils fixed at build time, gathered by the leaves) and steps it with a CellAdvance
(cpp/include/fv/CellAdvance.hpp:27-47). ``CellEngine`` is that pair on the device for a level-0 mesh: the leaves are given
as the mesh's arrays (level, ci, cj, ck) in the mesh's order, and states cross as (nleaf, 5) arrays in that order.

    eng = CellEngine(params, level, ci, cj, ck)      # CellFluxEngine(eos, riemann, muscl, bc) + build(mesh)
    eng.set_state(U)                                  # CellMesh::U
    R, s = eng.residual()                             # CellFluxEngine::residual(mesh, U, R)
    s = eng.step(dt, t)                               # CellAdvance::step(dt, t)

There is no CPU fallback: without the library or a device every call fails.
"""
import ctypes

import numpy as np

from . import params as P
from .runtime import FVG_ERR_ARGUMENT, FVG_ERR_CONFIG, FVG_OK, _dp, load_library


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def base_leaves(params, order="morton"):
    """The level-0 leaves of the base mesh of ``params`` as (level, ci, cj, ck) int32 arrays: in the reference's order
    (Morton key of (i, j, k), the CellMesh sort; cpp/include/fv/CellKey.hpp) or in row-major cell order ("rows")."""
    p = P.resolve(params)
    nx, ny, nz = int(p["nx"]), int(p["ny"]), int(p.get("nz", 1) or 1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel().astype(np.int64), j.ravel().astype(np.int64), k.ravel().astype(np.int64)
    if order == "morton":
        key = np.zeros_like(i)
        dim = 3 if nz > 1 else 2
        for b in range(21 if dim == 3 else 29):
            key |= ((i >> b) & 1) << (dim * b)
            key |= ((j >> b) & 1) << (dim * b + 1)
            if dim == 3:
                key |= ((k >> b) & 1) << (dim * b + 2)
        o = np.argsort(key, kind="stable")
        i, j, k = i[o], j[o], k[o]
    z = np.zeros(i.size, dtype=np.int32)
    return z, i.astype(np.int32), j.astype(np.int32), k.astype(np.int32)


class CellEngine:
    """CellFluxEngine + CellAdvance of a level-0 mesh on one GPU."""

    def __init__(self, params, level, ci, cj, ck=None, U=None, device=0):
        self.lib = load_library()
        self.params = P.resolve(params)
        self.cfg = P.to_config(self.params, precision=0, device=device)
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in (level, ci, cj, ck if ck is not None else np.zeros_like(ci))]
        self.level, self.ci, self.cj, self.ck = arrs
        self.nleaf = len(self.level)
        h = ctypes.c_void_p()
        rc = self.lib.fvg_cells_create(ctypes.byref(self.cfg), self.nleaf, *[_ip(a) for a in arrs], ctypes.byref(h))
        if rc != FVG_OK:
            msg = self.lib.fvg_create_error().decode()
            raise (ValueError if rc in (FVG_ERR_CONFIG, FVG_ERR_ARGUMENT) else RuntimeError)(f"fvg_cells_create: {msg}")
        self.h = h
        nl, nf = ctypes.c_longlong(), ctypes.c_longlong()
        self.lib.fvg_cells_info(h, ctypes.byref(nl), ctypes.byref(nf))
        self.nface = nf.value
        if U is not None:
            self.set_state(U)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fvg_cells_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc, what):
        if rc != FVG_OK:
            raise RuntimeError(f"fvg_cells_{what}: {self.lib.fvg_cells_last_error(self.h).decode()} (status {rc})")

    def _leaf_array(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != (self.nleaf, 5):
            raise ValueError(f"a state is a ({self.nleaf}, 5) float64 array")
        return a

    def set_state(self, U):
        U = self._leaf_array(U)
        self._check(self.lib.fvg_cells_upload_state(self.h, _dp(U), self.nleaf), "upload_state")

    def state(self, out=None):
        """The leaf state, into `out` if given (a C-contiguous (nleaf, 5) float64 array, e.g. in pinned memory)."""
        U = np.empty((self.nleaf, 5)) if out is None else out
        if U.shape != (self.nleaf, 5) or U.dtype != np.float64 or not U.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of shape ({self.nleaf}, 5)")
        self._check(self.lib.fvg_cells_download_state(self.h, _dp(U), self.nleaf), "download_state")
        return U

    def residual(self):
        """(R, largest face wave speed) of the state held."""
        R = np.empty((self.nleaf, 5))
        s = ctypes.c_double()
        self._check(self.lib.fvg_cells_residual(self.h, _dp(R), self.nleaf, ctypes.byref(s)), "residual")
        return R, s.value

    def step(self, dt, t=0.0):
        """One step of length dt (CellAdvance::step); the first stage's largest face wave speed."""
        s = ctypes.c_double()
        self._check(self.lib.fvg_cells_step(self.h, float(dt), float(t), ctypes.byref(s)), "step")
        return s.value

    def advance(self, dt, nsteps):
        """nsteps steps of length dt enqueued back to back; the last step's first-stage speed."""
        s = ctypes.c_double()
        self._check(self.lib.fvg_cells_advance(self.h, float(dt), int(nsteps), ctypes.byref(s)), "advance")
        return s.value

    def stream(self):
        v = ctypes.c_void_p()
        self._check(self.lib.fvg_cells_stream(self.h, ctypes.byref(v)), "stream")
        return v.value
