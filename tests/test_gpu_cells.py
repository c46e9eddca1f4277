"""The cell engine of an adaptive mesh on the GPU (fvg_cells_*, fenice_b200.cells) against the reference's own engine
(CellFluxEngine + CellAdvance compiled from its sources, oracle/_ref) on level-0 meshes, bit for bit: the matrices of the
reference's level-0 tests (cpp/tests/test_amr_octree_advance.cpp:70-108 in 3-D, cpp/tests/test_amr_mesh.cpp:440-531 in
2-D, cpp/tests/test_amr_octree_physics.cpp:54-92 for the 3-D viscous terms) -- boundary sets with walls, no-slip and moving walls, inlets, outlets, transmissive and periodic sides; first order,
MUSCL, WENO3-Z and WENO5-Z with boundary_order 1 and 2; Euler, SSP-RK2 and SSP-RK3 -- each advanced 4 steps of
dt = 2e-3 from a seeded smooth state on the reference rig's mesh (9 x 7 x 5 cells of 1.7 x 1.1 x 0.9), the CellMesh built
with max_level 0 and 2 (every leaf of level 0 either way). The residual is compared too, and with the uniform path's
(fvg_residual of the same cells), which the reference's tests require its engine to equal."""
import numpy as np
import pytest

import cases
from fenice_b200 import Run
from fenice_b200.cells import CellEngine, base_leaves
from oracle.oracle import Reference, ReferenceCells, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="the reference is not compiled (oracle/_ref)")]

RIG = dict(nx=9, ny=7, Lx=1.7, Ly=1.1, u_in=0.7, v_in=0.2, rho_in=1.2, p_out=1.3)
RIG3 = dict(RIG, nz=5, Lz=0.9)
SCHEMES = ["Explicit Euler", "SSP Runge-Kutta 2", "SSP Runge-Kutta 3"]
# (reconstruction, boundary_order, time schemes)
RECON = [("none", 1, SCHEMES), ("muscl", 1, SCHEMES), ("muscl", 2, SCHEMES), ("weno3", 1, SCHEMES[2:]), ("weno3", 2, SCHEMES[2:]),
         ("weno5", 1, SCHEMES[2:]), ("weno5", 2, SCHEMES[2:])]
SETS3 = [("wall", "outlet", "no_slip", "moving_wall", "transmissive", "wall"), ("periodic", "periodic", "wall", "wall", "transmissive", "no_slip"),
         ("vel_inlet", "transmissive", "periodic", "periodic", "periodic", "periodic")]
SETS2 = [("wall", "outlet", "no_slip", "moving_wall"), ("periodic", "periodic", "wall", "wall"), ("transmissive", "vel_inlet", "periodic", "periodic")]


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def params_of(rig, bc, recon, order, scheme, **extra):
    p = dict(rig, reconstruction=recon, boundary_order=order, time_scheme=scheme, muscl_limiter="Van Leer")
    p.update(extra)
    names = ("bc_xmin", "bc_xmax", "bc_ymin", "bc_ymax", "bc_zmin", "bc_zmax")
    p.update(dict(zip(names, bc)))
    if len(bc) == 4:
        p["bc_zmin"] = p["bc_zmax"] = "periodic"
    return p


def leaf_state(params, seed, rc):
    """A seeded smooth state of the base mesh, in the order of the leaves rc.ci / cj / ck."""
    nx, ny, nz = params["nx"], params["ny"], params.get("nz", 1)
    U = cases.smooth_field(nx, ny, nz, seed=seed)
    return U, U[(rc.ck.astype(np.int64) * ny + rc.cj) * nx + rc.ci]


def compare(params, seed, max_levels=(0, 2), steps=4, dt=2e-3):
    ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
    for ml in max_levels:
        rc = ReferenceCells(ref, ml)
        assert np.all(rc.level == 0)
        _, Ul = leaf_state(params, seed, rc)
        rc.set_state(Ul)
        eng = CellEngine(params, rc.level, rc.ci, rc.cj, rc.ck, U=Ul)
        assert eng.nface == rc.nface
        R_ref, s_ref = rc.residual()
        R, s = eng.residual()
        assert bits_equal(R, R_ref) and s == s_ref, (ml, np.abs(R - R_ref).max(), s, s_ref)
        s_refs = rc.steps(dt, steps)
        for k in range(steps):
            sk = eng.step(dt, k * dt)
            assert sk == s_refs[k], (ml, k, sk, s_refs[k])
        assert bits_equal(eng.state(), rc.state()), (ml, np.abs(eng.state() - rc.state()).max())
        eng.close()
        del rc


@pytest.mark.parametrize("bc", SETS3, ids=["/".join(b) for b in SETS3])
@pytest.mark.parametrize("recon,order,schemes", RECON, ids=[f"{r}_bo{o}" for r, o, _ in RECON])
def test_level0_octree_steps_match_the_reference(bc, recon, order, schemes):
    for sc in schemes:
        compare(params_of(RIG3, bc, recon, order, sc), seed=31)


@pytest.mark.parametrize("big", [0, 1])
@pytest.mark.parametrize("bc", SETS2, ids=["/".join(b) for b in SETS2])
@pytest.mark.parametrize("recon,order,schemes", RECON, ids=[f"{r}_bo{o}" for r, o, _ in RECON])
def test_level0_quadtree_steps_match_the_reference(bc, recon, order, schemes, big):
    rig = dict(RIG, nx=96, ny=64) if big else RIG
    for sc in schemes:
        compare(params_of(rig, bc, recon, order, sc), seed=32 + big, max_levels=(0,) if big else (0, 2))


@pytest.mark.parametrize("name,params,uniform", [
    ("weno5_lowmach_3d", params_of(RIG3, SETS3[0], "weno5", 2, SCHEMES[2], riemann_solver="lowmach"), True),
    ("muscl_mc_stiffened_2d", dict(params_of(RIG, SETS2[1], "muscl", 2, SCHEMES[1]), muscl_limiter="MC", eos_type="Stiffened Gas", gamma=4.4, p_inf=3.0), True),
    ("weno5_noblend_1row", dict(params_of(dict(RIG, nx=40, ny=1), ("transmissive",) * 4, "weno5", 2, SCHEMES[2]), shock_blend=0.0), True),
    # periodic axes of fewer cells than WENO5-Z's three: the cell engine wraps the whole stencil, the uniform solver makes
    # those periodic faces a first-order seam (its wrap halo needs n >= 3, cpp/src/Simulation.cpp:869-885); the two differ
    # there in the reference too, so only the reference's engine is the check
    ("weno5_thin_periodic", params_of(dict(RIG3, nx=3, ny=2, nz=4), ("periodic",) * 6, "weno5", 2, SCHEMES[2]), False),
])
def test_residual_matches_the_reference_and_the_uniform_path(name, params, uniform):
    ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
    rc = ReferenceCells(ref, 0)
    Urows, Ul = leaf_state(params, 40, rc)
    rc.set_state(Ul)
    eng = CellEngine(params, rc.level, rc.ci, rc.cj, rc.ck, U=Ul)
    R, s = eng.residual()
    R_ref, s_ref = rc.residual()
    assert bits_equal(R, R_ref) and s == s_ref
    if not uniform:
        eng.close()
        return
    run = Run(params, U=Urows)
    Ru, su = run.residual(Urows)
    nx, ny = params["nx"], params["ny"]
    assert bits_equal(R, Ru[(rc.ck.astype(np.int64) * ny + rc.cj) * nx + rc.ci]) and s == su
    run.close()
    eng.close()


def test_leaf_order_is_free():
    """The engine takes the leaves in any order: the same cells listed row by row give the same states, leaf for leaf."""
    params = params_of(RIG3, SETS3[0], "weno5", 2, SCHEMES[2])
    lv, ci, cj, ck = base_leaves(params, "morton")
    lr, ri, rj, rk = base_leaves(params, "rows")
    U = cases.smooth_field(9, 7, 5, seed=50)
    a = CellEngine(params, lv, ci, cj, ck, U=U[(ck.astype(np.int64) * 7 + cj) * 9 + ci])
    b = CellEngine(params, lr, ri, rj, rk, U=U)
    for k in range(3):
        assert a.step(2e-3, k * 2e-3) == b.step(2e-3, k * 2e-3)
    Ua = np.empty_like(U)
    Ua[(ck.astype(np.int64) * 7 + cj) * 9 + ci] = a.state()
    assert bits_equal(Ua, b.state())


VSETS = [("moving_wall", "no_slip", "wall", "moving_wall", "no_slip", "moving_wall"), ("no_slip", "moving_wall", "moving_wall", "wall", "moving_wall", "wall"),
         ("wall", "transmissive", "no_slip", "moving_wall", "periodic", "periodic"), ("periodic", "periodic", "moving_wall", "no_slip", "wall", "moving_wall"),
         ("outlet", "vel_inlet", "periodic", "periodic", "no_slip", "moving_wall"), ("periodic",) * 6]
VRECON = [("none", 1), ("muscl", 1), ("muscl", 2), ("weno3", 2), ("weno5", 2)]


@pytest.mark.parametrize("bc", VSETS, ids=["/".join(b) for b in VSETS])
@pytest.mark.parametrize("recon,order", VRECON, ids=[f"{r}_bo{o}" for r, o in VRECON])
def test_viscous_level0_octree_matches_the_reference(bc, recon, order):
    """The 3-D viscous terms (every wall rule, moving walls on every axis, boundary_order 1 and 2, mu small and large so the
    viscous speed bound wins in some cases): residual and speed bit for bit against the reference's engine and the uniform
    path, then 4 SSP-RK3 steps against CellAdvance."""
    for mu in (0.02, 0.6):
        params = params_of(RIG3, bc, recon, order, SCHEMES[2], use_viscous=True, mu=mu, pr=0.72)
        ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
        rc = ReferenceCells(ref, 0)
        Urows, Ul = leaf_state(params, 60, rc)
        rc.set_state(Ul)
        eng = CellEngine(params, rc.level, rc.ci, rc.cj, rc.ck, U=Ul)
        R, s = eng.residual()
        R_ref, s_ref = rc.residual()
        assert bits_equal(R, R_ref) and s == s_ref, (mu, np.abs(R - R_ref).max(), s, s_ref)
        run = Run(params, U=Urows)
        Ru, su = run.residual(Urows)
        nx, ny = params["nx"], params["ny"]
        assert bits_equal(R, Ru[(rc.ck.astype(np.int64) * ny + rc.cj) * nx + rc.ci]) and s == su
        run.close()
        s_refs = rc.steps(2e-3, 4)
        for k in range(4):
            assert eng.step(2e-3, k * 2e-3) == s_refs[k]
        assert bits_equal(eng.state(), rc.state())
        eng.close()


VSETS2 = [("moving_wall", "no_slip", "wall", "moving_wall"), ("periodic", "periodic", "moving_wall", "no_slip"), ("wall", "outlet", "periodic", "periodic"),
          ("no_slip", "vel_inlet", "moving_wall", "transmissive")]


@pytest.mark.parametrize("bc", VSETS2, ids=["/".join(b) for b in VSETS2])
@pytest.mark.parametrize("recon,order", VRECON, ids=[f"{r}_bo{o}" for r, o in VRECON])
def test_viscous_level0_quadtree_matches_the_reference(bc, recon, order):
    """The 2-D viscous terms (cell_quantities / viscous_fluxes of a quadtree): residual and speed bit for bit against the
    reference's engine, then 4 SSP-RK3 steps against CellAdvance; mu small and large."""
    for mu in (0.02, 0.6):
        params = params_of(RIG, bc, recon, order, SCHEMES[2], use_viscous=True, mu=mu, pr=0.72)
        compare(params, seed=70, max_levels=(0,))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("recon,order", [("muscl", 2), ("weno5", 2), ("none", 1)])
def test_body_force_level0_matches_the_reference(dim, recon, order):
    """The body force (ConstantBodyForce on every axis, after the viscous terms in 3-D), bit for bit."""
    rig = RIG3 if dim == 3 else RIG
    bc = SETS3[0] if dim == 3 else SETS2[0]
    extra = dict(use_bodyforce=True, gx=0.3, gy=-0.7, gz=0.2)
    if dim == 3:
        extra.update(use_viscous=True, mu=0.05, pr=0.72)
    compare(params_of(rig, bc, recon, order, SCHEMES[2], **extra), seed=80, max_levels=(0,))


@pytest.mark.parametrize("visc", [False, True], ids=["inviscid", "viscous"])
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("bc", SETS3, ids=["/".join(b) for b in SETS3])
def test_hancock_level0_octree_matches_the_reference(bc, order, visc):
    """MUSCL-Hancock on a level-0 octree (cpp/tests/test_amr_octree_advance.cpp:110-152): the leaves' limited side states
    predicted by half a step, the Riemann problems on them, bit for bit against CellAdvance for 4 steps."""
    extra = dict(use_viscous=True, mu=0.02, pr=0.72) if visc else {}
    compare(params_of(RIG3, bc, "muscl", order, "MUSCL-Hancock", **extra), seed=90)


@pytest.mark.parametrize("bc", SETS2, ids=["/".join(b) for b in SETS2])
def test_hancock_level0_quadtree_matches_the_reference(bc):
    for order in (1, 2):
        compare(params_of(RIG, bc, "muscl", order, "MUSCL-Hancock", muscl_limiter="MC"), seed=91)
        compare(params_of(dict(RIG, nx=96, ny=64), bc, "muscl", order, "MUSCL-Hancock"), seed=92, max_levels=(0,))


def test_hancock_body_force_level0_matches_the_reference():
    for rig, bc in ((RIG3, SETS3[1]), (RIG, SETS2[0])):
        compare(params_of(rig, bc, "muscl", 2, "MUSCL-Hancock", use_bodyforce=True, gx=0.3, gy=-0.7, gz=0.2), seed=93, max_levels=(0,))
