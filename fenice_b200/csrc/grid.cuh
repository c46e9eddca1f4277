// The mesh, its boundary conditions and the device-side control block of a run.
//
// HBM layout: the conservative state is stored as NV planes (structure of arrays), NV = 4 on a 2-D mesh
// ([rho, rho u, rho v, rho E]; the reference's rho w is identically +0 there) and 5 on a 3-D mesh; plane q of
// cell (i, j, k) is at q * plane + (k * ny + j) * nx + i, the reference's row-major cell order
// (cpp/include/fv/Core.hpp:114). `plane` is the cell count rounded up to 32 so every plane starts on a 256-byte
// boundary.
#pragma once

#include "physics.cuh"

namespace fvg {

// boundary types, in the order of the reference's BCType (cpp/include/fv/Boundaries.hpp:15)
constexpr int kBcWall = 0, kBcNoSlip = 1, kBcMovingWall = 2, kBcVelInlet = 3, kBcMassflowInlet = 4, kBcOutlet = 5,
              kBcTransmissive = 6, kBcPeriodic = 7, kBcNonReflecting = 8;
// what lies beyond a side for the reconstruction stencil (cpp/src/Simulation.cpp:868-905): nothing (edge
// replication, first-order boundary faces), the periodic wrap, or the ghost slab of the boundary condition; and, for
// one part of a slab-decomposed mesh, the neighbouring part's cells, held in ghost planes beyond the side (the state
// arrays of a part are allocated with Bc::ext planes there, so indices -ext .. -1 and n .. n + ext - 1 are real cells)
constexpr int kHaloNone = 0, kHaloWrap = 1, kHaloSlab = 2, kHaloPeer = 3;

// Device control block of a run: the clock, the step and the wave speeds, all on the device so a step needs no
// host round trip (and can be captured in a CUDA graph).
struct Ctl {
    double t, t_end, dt, dt_max, cfl, L;
    double s_lag;       // MUSCL-Hancock: wave speed of the previous step (0: none yet)
    double s_step;      // largest wave speed of the current step
    double s_stage[3];  // wave speed of each stage of the step
    double half_dt;     // MUSCL-Hancock: half the step the predictor advances the face states by
    double stage_t;     // the time of the residual being taken (TimeScheme::stage_time)
    int active;         // this step runs (t < t_end, steps < max_steps, no error)
    int seed;           // MUSCL-Hancock: this step first takes one plain residual for the wave speed
    int always;         // 1: the gate of calls outside the time loop
    int steps, max_steps;
    int status;         // 0 ok; 1 the solution diverged (non-finite speed or dt, or t no longer advances); 3 a
                        // time-dependent boundary value was not finite, or rho_in or p_out not positive, at a stage time;
                        // 5 a TMA copy of a stage tile, 6 a tensor-core step of the sensor did not complete (a bounded wait gave up)
};

struct Mesh {
    int nx, ny, nz;
    long long ncells, plane;
    double dx, dy, dz;
    double area[3];   // face areas used by the balance: 2-D (dy, dx); 3-D (dy dz, dx dz, dx dy)
    double inv_cell;  // 1 / cell area (2-D) or 1 / cell volume (3-D)
};

struct Bc {
    int type[6];   // left, right, bottom, top, front, back
    int halo[6];   // kHalo* of each side for the reconstruction stencil
    double u_in, v_in, p_out;
    // immersed body (null without one): the solid mask, and the forced states the residual reads in place of the cells'
    // own (ghost cells filled from their image points, deeper solid cells at rest): slot[c] >= 0 -> forced[5 slot + q]
    const unsigned char* solid;
    const int* slot;
    const double* forced;
    // the constant body force (gz = 0 on a 2-D mesh), on when grav_on
    double grav[3];
    int grav_on;
    // planes of the neighbouring part held beyond each side (kHaloPeer sides only; 0 elsewhere)
    int ext[6];
    // mass-flow inlets: the target velocity of each side for the residual being taken (device array of 6, written from
    // the residual's state before it; null without a mass-flow side)
    const double* u_target;
    // non-reflecting outlets: relaxation sigma, transverse weight beta (< 0: the local Mach number), the domain length
    // and the cell size per axis
    double nrbc_sigma, nrbc_beta, length[3], h[3];
    // time-dependent boundary values [u_in, v_in, rho_in, p_out] at the stage time of the residual being taken (device
    // array of 4, written before it); null when they are the constants above
    const double* tv;
    // the case's source terms S (planes in the state's layout, the state's ghost planes included) added to the
    // residual; null without
    const double* src;
};

__device__ __forceinline__ double bc_u_in(const Bc& bc) { return bc.tv ? bc.tv[0] : bc.u_in; }
__device__ __forceinline__ double bc_v_in(const Bc& bc) { return bc.tv ? bc.tv[1] : bc.v_in; }
__device__ __forceinline__ double bc_p_out(const Bc& bc) { return bc.tv ? bc.tv[3] : bc.p_out; }

// Whether position g along an axis of n cells is a cell whose state is in the arrays (a cell of the mesh, or of a
// neighbouring part's ghost planes beyond a kHaloPeer side), and the wrapped index of a periodic axis otherwise.
template <bool FULL = true> __device__ __forceinline__ bool held(const Bc& bc, int axis, int g, int n) {
    if constexpr (!FULL) return g >= 0 && g < n;
    return (g >= 0 && g < n) || (g < 0 && bc.halo[2 * axis] == kHaloPeer && g >= -bc.ext[2 * axis]) ||
           (g >= n && bc.halo[2 * axis + 1] == kHaloPeer && g < n + bc.ext[2 * axis + 1]);
}

// BoundaryManager::ghost_state (cpp/src/Boundaries.cpp:106-153) for the sides a device run supports (every type but
// the non-reflecting outlet, which needs more than one cell; the mass-flow inlet's target comes from Bc::u_target).
template <typename T, int NV>
__device__ __forceinline__ St<T, NV> ghost_state(const Eos<T>& e, const Bc& bc, int side, const St<T, NV>& Ui) {
    const int type = bc.type[side];
    if (type == kBcTransmissive) return Ui;
    const int axis = side >> 1;
    const T nxn = axis == 0 ? T(1) : T(0), nyn = axis == 1 ? T(1) : T(0), nzn = axis == 2 ? T(1) : T(0);
    const St<T, NV> Wi = c2p(e, Ui);
    St<T, NV> Wg = Wi;
    const T wi = NV == 5 ? Wi[NV - 1] : T(0);   // the z velocity (+0 on a planar mesh, as in the reference)
    switch (type) {
    case kBcWall: {
        const T Vn = Wi[1] * nxn + Wi[2] * nyn + wi * nzn;
        Wg[1] = Wi[1] - T(2) * Vn * nxn;
        Wg[2] = Wi[2] - T(2) * Vn * nyn;
        if constexpr (NV == 5) Wg[4] = Wi[4] - T(2) * Vn * nzn;
        break;
    }
    case kBcNoSlip:
        Wg[1] = -Wi[1];
        Wg[2] = -Wi[2];
        if constexpr (NV == 5) Wg[4] = -Wi[4];
        break;
    case kBcMovingWall:
    case kBcVelInlet:
        Wg[1] = T(2) * T(bc_u_in(bc)) - Wi[1];
        Wg[2] = T(2) * T(bc_v_in(bc)) - Wi[2];
        if constexpr (NV == 5) Wg[4] = -Wi[4];
        break;
    case kBcMassflowInlet:   // the x velocity of the side's mass-flow target, whatever the side's axis (as the reference)
        Wg[1] = T(2) * T(bc.u_target[side]) - Wi[1];
        Wg[2] = T(2) * T(bc_v_in(bc)) - Wi[2];
        if constexpr (NV == 5) Wg[4] = -Wi[4];
        break;
    case kBcOutlet: {
        const T Vn = Wi[1] * nxn + Wi[2] * nyn + wi * nzn;
        const bool outflow = Vn >= T(0);
        Wg[1] = outflow ? Wi[1] : T(0);
        Wg[2] = outflow ? Wi[2] : T(0);
        if constexpr (NV == 5) Wg[4] = outflow ? Wi[4] : T(0);
        Wg[3] = vmax(T(bc_p_out(bc)), T(1e-5));
        break;
    }
    default: break;
    }
    return p2c(e, Wg);
}

template <int NV> __device__ __forceinline__ St<double, NV> read_cell(const double* __restrict__ U, long long plane, long long c) {
    St<double, NV> s;
#pragma unroll
    for (int q = 0; q < NV; ++q) s[q] = U[q * plane + c];
    return s;
}

// The state a residual reads for cell c: the cell's own, or its forced state where the immersed body overrides it
// (ImmersedBoundary::force_in_place, cpp/src/Physics.cpp:962-973: the residual sees the forced field; the update does not).
template <int NV> __device__ __forceinline__ St<double, NV> read_state(const Bc& bc, const double* __restrict__ U, long long plane, long long c) {
    if (bc.slot) {
        const int s = bc.slot[c];
        if (s >= 0) {
            St<double, NV> f;
#pragma unroll
            for (int q = 0; q < NV; ++q) f[q] = bc.forced[5 * (long long)s + q];
            return f;
        }
    }
    return read_cell<NV>(U, plane, c);
}

// ConstantBodyForce::add_to (cpp/src/Physics.cpp:832-844) for one cell of state u, into r in its order:
// r1 += rho gx, r2 += rho gy, r3 += m_x gx + m_y gy, then with gz != 0 (a 3-D mesh) r3 += m_z gz and r4 += rho gz.
// RhsSourceTerms' expression source (Simulation.cpp:397-412, add_source): r[q] += S[q] of the cell.
template <int NV> __device__ __forceinline__ void add_source(const Bc& bc, long long plane, long long cell, St<double, NV>& r) {
#pragma unroll
    for (int q = 0; q < NV; ++q) r[q] = r[q] + bc.src[q * plane + cell];
}

template <int NV> __device__ __forceinline__ void add_body_force(const Bc& bc, const St<double, NV>& u, St<double, NV>& r) {
    const double gx = bc.grav[0], gy = bc.grav[1], gz = bc.grav[2];
    r[1] = r[1] + u[0] * gx;
    r[2] = r[2] + u[0] * gy;
    r[3] = r[3] + (u[1] * gx + u[2] * gy);
    if constexpr (NV == 5) {
        if (gz != 0.0) {
            r[3] = r[3] + u[4] * gz;
            r[4] = r[4] + u[0] * gz;
        }
    }
}

// The conservative state at cell position (i, j, k) of the reconstruction stencil, which may lie outside the mesh along
// one axis: the periodic wrap, the ghost-slab state of the mirrored cell (fill_ghost_slab, cpp/src/Boundaries.cpp:202-228:
// layer l beyond the side is ghost_state of the interior cell l cells from it), or edge replication (pad_primitives,
// cpp/src/Schemes.cpp:915-969). Positions outside along two axes (never on a stencil of a face of the mesh) and those of a
// tile that overhangs the mesh are clamped, so every read is inside the state arrays.
//
// FULL = false: a run without part interfaces (no kHaloPeer side), for the hot kernels (the interface test and the
// ghost-plane clamp compiled out).
template <int DIM, int NV, bool FULL = true>
__device__ __forceinline__ St<double, NV> stencil_cons(const Mesh& m, const Bc& bc, const Eos<double>& e, const double* __restrict__ U, int i, int j,
                                                       int k) {
    int idx[3] = {i, j, k};
    const int n3[3] = {m.nx, m.ny, m.nz};
    int out_axis = -1, nout = 0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        const bool lo = idx[a] < 0, hi = idx[a] >= n3[a];
        if (!lo && !hi) continue;
        const int kind = bc.halo[2 * a + (hi ? 1 : 0)];
        if (kind == kHaloWrap) {
            idx[a] = ((idx[a] % n3[a]) + n3[a]) % n3[a];
            continue;
        }
        if (FULL && kind == kHaloPeer) continue;   // the neighbouring part's cell (clamped below onto its ghost planes)
        out_axis = a;
        ++nout;
    }
    // every index onto the cells the arrays hold (a part's ghost planes included); positions beyond them belong to a
    // tile overhanging the mesh or the part, whose results are discarded
    const auto clamp_held = [&]() {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int lo = FULL ? -bc.ext[2 * a] : 0, hi = FULL ? n3[a] - 1 + bc.ext[2 * a + 1] : n3[a] - 1;
            idx[a] = idx[a] < lo ? lo : (idx[a] > hi ? hi : idx[a]);
        }
    };
    if (nout == 1) {
        const int a = out_axis;
        const bool hi = idx[a] >= n3[a];
        const int side = 2 * a + (hi ? 1 : 0);
        if (bc.halo[side] == kHaloSlab) {
            int l = hi ? idx[a] - n3[a] : -1 - idx[a];
            l = l < n3[a] ? l : n3[a] - 1;
            idx[a] = hi ? n3[a] - 1 - l : l;
            // the other axes too: beyond a part interface a position may lie past the ghost planes (a tile overhanging
            // the part), and reading it would leave the state arrays
            clamp_held();
            const long long c = ((long long)idx[2] * m.ny + idx[1]) * m.nx + idx[0];
            return ghost_state(e, bc, side, read_state<NV>(bc, U, m.plane, c));
        }
    }
    clamp_held();
    const long long c = ((long long)idx[2] * m.ny + idx[1]) * m.nx + idx[0];
    return read_state<NV>(bc, U, m.plane, c);
}

// Solidity of a stencil position for WENO5-Z's narrow stencil beside an immersed body (make_grid, cpp/src/Schemes.cpp:
// 1004-1019): a position outside the mesh is solid if the cell edge replication puts there, or the cell a periodic wrap
// puts there, is solid.
template <int DIM> __device__ __forceinline__ unsigned char stencil_solid(const Mesh& m, const Bc& bc, int i, int j, int k) {
    const int n3[3] = {m.nx, m.ny, m.nz};
    const int p[3] = {i, j, k};
    int c[3], w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        c[a] = p[a] < 0 ? 0 : (p[a] >= n3[a] ? n3[a] - 1 : p[a]);
        w[a] = ((p[a] % n3[a]) + n3[a]) % n3[a];
    }
    const long long cc = ((long long)c[2] * m.ny + c[1]) * m.nx + c[0], cw = ((long long)w[2] * m.ny + w[1]) * m.nx + w[0];
    return (bc.solid[cc] != 0 || bc.solid[cw] != 0) ? 1 : 0;
}

// BoundaryManager::nonreflecting_ghost (cpp/src/Boundaries.cpp:155-191) of the cell (i, j, k) next to side `side`, with
// its tangential neighbours as apply_side gathers them (Boundaries.cpp:316-355): along each other axis of more than one
// cell, the cells on either side (wrapped on a periodic axis, a neighbouring part's across a part interface, else the cell
// itself at an end, which halves the span). The ghost differs from the cell in the incoming acoustic characteristic only.
template <int NV>
__device__ __forceinline__ St<double, NV> nrbc_ghost(const Mesh& m, const Bc& bc, const Eos<double>& e, const double* __restrict__ U, int side, int i,
                                                     int j, int k, const St<double, NV>& Ui) {
    const int axis = side >> 1;
    const double s = (side & 1) ? 1.0 : -1.0;
    const int mom[3] = {1, 2, NV == 5 ? 4 : 1};
    const St<double, NV> Wi = c2p(e, Ui);
    St<double, NV> Wg = Wi;
    const int qv = mom[axis];
    const double u_out = s * Wi[qv];
    const double c = sound_speed(e, Wi[3], Wi[0]);
    const double M = vmin(vmax(u_out / c, -1.0), 1.0);
    if (M >= 1.0) return p2c(e, Wg);   // supersonic outflow: nothing enters
    const double h = bc.h[axis];
    const double K = bc.nrbc_sigma * c * (1.0 - M * M) / bc.length[axis];
    const double beta = bc.nrbc_beta >= 0.0 ? bc.nrbc_beta : fabs(M);
    double T1 = 0.0;
    if (beta < 1.0) {
        const int n3[3] = {m.nx, m.ny, m.nz};
        const int ijk[3] = {i, j, k};
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            if (t == axis || n3[t] == 1) continue;
            const bool peer_lo = bc.halo[2 * t] == kHaloPeer, peer_hi = bc.halo[2 * t + 1] == kHaloPeer;
            const bool wrap = bc.type[2 * t] == kBcPeriodic && bc.type[2 * t + 1] == kBcPeriodic && !peer_lo && !peer_hi;
            int lo = ijk[t] - 1, hi = ijk[t] + 1;
            double span = 2.0;
            if (wrap) {
                lo = (lo + n3[t]) % n3[t];
                hi = hi % n3[t];
            } else {
                if (lo < 0 && !peer_lo) {
                    lo = 0;
                    span -= 1.0;
                }
                if (hi >= n3[t] && !peer_hi) {
                    hi = n3[t] - 1;
                    span -= 1.0;
                }
                if (span <= 0.0) continue;
            }
            int a[3] = {i, j, k}, b[3] = {i, j, k};
            a[t] = lo;
            b[t] = hi;
            const St<double, NV> Wl = c2p(e, read_state<NV>(bc, U, m.plane, ((long long)a[2] * m.ny + a[1]) * m.nx + a[0]));
            const St<double, NV> Wh = c2p(e, read_state<NV>(bc, U, m.plane, ((long long)b[2] * m.ny + b[1]) * m.nx + b[0]));
            const double ht = span * bc.h[t];
            const int qt = mom[t];
            T1 += Wi[qt] * (Wh[3] - Wl[3]) / ht + Wi[0] * c * c * (Wh[qt] - Wl[qt]) / ht - Wi[0] * c * s * Wi[qt] * (Wh[qv] - Wl[qv]) / ht;
        }
    }
    const double dw1 = -h * (K * (Wi[3] - bc_p_out(bc)) - (1.0 - beta) * T1) / (c - u_out);
    Wg[3] = Wi[3] + 0.5 * dw1;
    Wg[qv] = Wi[qv] - s * dw1 / (2.0 * Wi[0] * c);
    Wg[0] = Wi[0] + 0.5 * dw1 / (c * c);
    return p2c(e, Wg);
}

// The first-order ghost of the cell (i, j, k) next to a side without a halo: ghost_state, or the non-reflecting ghost.
template <int NV, bool FULL = true>
__device__ __forceinline__ St<double, NV> side_ghost(const Mesh& m, const Bc& bc, const Eos<double>& e, const double* __restrict__ U, int side, int i,
                                                     int j, int k) {
    const St<double, NV> Ui = read_state<NV>(bc, U, m.plane, ((long long)k * m.ny + j) * m.nx + i);
    if (FULL && bc.type[side] == kBcNonReflecting) return nrbc_ghost<NV>(m, bc, e, U, side, i, j, k, Ui);
    return ghost_state(e, bc, side, Ui);
}

// The first-order states of a boundary face whose side has no halo (BoundaryManager::apply_side,
// cpp/src/Boundaries.cpp:277-373): the cell next to the side and its ghost (the opposite cell on a periodic side).
// (FULL = false: a run without non-reflecting sides, the characteristic ghost compiled out)
template <int NV, bool FULL = true>
__device__ __forceinline__ void side_states(const Mesh& m, const Bc& bc, const Eos<double>& e, const double* __restrict__ U, int side, int i, int j, int k,
                                            St<double, NV>& UL, St<double, NV>& UR) {
    const long long c = ((long long)k * m.ny + j) * m.nx + i;
    const St<double, NV> Ui = read_state<NV>(bc, U, m.plane, c);
    St<double, NV> Ug;
    if (bc.type[side] == kBcPeriodic) {
        int idx[3] = {i, j, k};
        const int a = side >> 1, n = a == 0 ? m.nx : (a == 1 ? m.ny : m.nz);
        idx[a] = (side & 1) ? idx[a] - (n - 1) : idx[a] + (n - 1);
        Ug = read_state<NV>(bc, U, m.plane, ((long long)idx[2] * m.ny + idx[1]) * m.nx + idx[0]);
    } else if (FULL && bc.type[side] == kBcNonReflecting) {
        Ug = nrbc_ghost<NV>(m, bc, e, U, side, i, j, k, Ui);
    } else {
        Ug = ghost_state(e, bc, side, Ui);
    }
    if (side & 1) {
        UL = Ui;
        UR = Ug;
    } else {
        UL = Ug;
        UR = Ui;
    }
}

// Warp and block maximum of a wave speed with the reference's rule `if (s > local) local = s` (a NaN never wins).
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        if (w > v) v = w;
    }
    return v;
}

// the cache line of a global address towards L2 (a hint: no completion, no fault on an address the kernel owns)
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

template <int NT> __device__ __forceinline__ double block_max(double v, double* red) {
    v = warp_max(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NW = (NT + 31) / 32;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
        r = red[0];
        for (int w = 1; w < NW; ++w)
            if (red[w] > r) r = red[w];
    }
    return r;
}

}   // namespace fvg
