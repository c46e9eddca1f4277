// The immersed body on the device: the forced states a residual reads, and the per-step reset of the solid cells
// (ImmersedBoundary::fill_ghosts_part / fill_ghost_cells, cpp/src/Physics.cpp:1539-1637, for a static body). The tables
// come from ibm_host.h. Every ghost state is computed from fluid cells only (solid interpolation cells weigh 0 and are not
// read), so the cells can be filled in any order, in place.
#pragma once

#include "grid.cuh"

namespace fvg {

struct IbmArgs {
    Mesh m;
    Eos<double> eos;
    int slip;                 // slip wall (inviscid) or no-slip
    int ng, nd;               // ghost cells, deep solid cells
    const int* ghost;         // [ng] cell
    const int* img_cell;      // [8 ng]
    const double* img_w;      // [8 ng]
    const double* ratio;      // [ng]
    const double* gn;         // [3 ng] wall normal (x, y, z)
    const int* deep;          // [nd] cell
    double rho_ref, p_ref;
    // a moving body: the wall velocity at each ghost's wall point [3 ng] and the velocity of each deep cell [3 nd]
    // (ImmersedBoundary::body_velocity); null for a static body
    const double* gvel;
    const double* dvel;
    // gravity (the body force): the ghost pressure carries the hydrostatic difference from the image point (per ghost its
    // span, ghost-wall + wall-image); hydro = 0 without
    int hydro;
    double grav[3];
    const double* span;
    const double* U;          // the state the ghost cells are filled from
    double* forced;           // force: [5 (ng + nd)] the forced states, by slot (ghosts first, then the deep cells)
    double* Uout;             // reset: the state written in place (may be U)
    int reset;                // 0: force (ghosts, deep cells at rest); 1: reset (ghosts, deep cells at the reference state)
    const int* gate;
};

template <int NV> __global__ void ibm_fill_kernel(const IbmArgs a) {
    if (!*a.gate) return;
    const int n = a.ng + a.nd;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        St<double, NV> out;
        long long cell;
        if (k < a.ng) {
            cell = a.ghost[k];
            // Probe::at (Physics.cpp:1053-1061): sum of w * cons_to_prim(cell) over the interpolation cells with w != 0
            double W[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            for (int q = 0; q < 8; ++q) {
                const double w = a.img_w[8 * k + q];
                if (w == 0.0) continue;
                const St<double, NV> Wq = c2p(a.eos, read_cell<NV>(a.U, a.m.plane, a.img_cell[8 * k + q]));
#pragma unroll
                for (int v = 0; v < NV; ++v) W[v] += w * Wq[v];
            }
            const double nx = a.gn[3 * k], ny = a.gn[3 * k + 1], nz = a.gn[3 * k + 2], ratio = a.ratio[k];
            // the hydrostatic pressure from the image point to the ghost cell (Physics.cpp:1592); W[3] is the pressure in both
            // layouts
            if (a.hydro) W[3] -= W[0] * a.span[k] * (a.grav[0] * nx + a.grav[1] * ny + (NV == 5 ? a.grav[2] * nz : 0.0));
            // in 2-D the reference's velocity index 4 is the z component, here the last of 4 is the pressure
            const double wz = NV == 5 ? W[4] : 0.0;
            const double un = NV == 5 ? W[1] * nx + W[2] * ny + wz * nz : W[1] * nx + W[2] * ny;
            double ux, uy, uz = 0.0;
            if (a.gvel) {   // a moving wall: the condition in the frame of the wall point (relative velocity reflected / through zero)
                const double wu = a.gvel[3 * k], wv = a.gvel[3 * k + 1], ww = a.gvel[3 * k + 2];
                const double ru = W[1] - wu, rv = W[2] - wv, rw = NV == 5 ? wz - ww : 0.0;
                const double rn = NV == 5 ? ru * nx + rv * ny + rw * nz : ru * nx + rv * ny;
                if (a.slip) {
                    ux = wu + ru - rn * nx - ratio * rn * nx;
                    uy = wv + rv - rn * ny - ratio * rn * ny;
                    if (NV == 5) uz = ww + rw - rn * nz - ratio * rn * nz;
                } else {
                    ux = wu - ratio * ru;
                    uy = wv - ratio * rv;
                    if (NV == 5) uz = ww - ratio * rw;
                }
            } else if (a.slip) {   // tangential velocity kept, normal velocity reflected through zero at the wall
                ux = W[1] - un * nx - ratio * un * nx;
                uy = W[2] - un * ny - ratio * un * ny;
                if (NV == 5) uz = wz - un * nz - ratio * un * nz;
            } else {        // the whole velocity through zero at the wall
                ux = -ratio * W[1];
                uy = -ratio * W[2];
                if (NV == 5) uz = -ratio * wz;
            }
            St<double, NV> Wg;
            Wg[0] = W[0];
            Wg[1] = ux;
            Wg[2] = uy;
            Wg[3] = W[3];
            if constexpr (NV == 5) Wg[4] = uz;
            out = p2c(a.eos, Wg);
        } else {
            cell = a.deep[k - a.ng];
            // at rest, or riding with a moving body
            const double* bv = a.dvel ? a.dvel + 3 * (long long)(k - a.ng) : nullptr;
            const double bu = bv ? bv[0] : 0.0, bvv = bv ? bv[1] : 0.0, bw = bv ? bv[2] : 0.0;
            St<double, NV> W;
            if (a.reset) {
                W[0] = a.rho_ref;
                W[1] = bu;
                W[2] = bvv;
                W[3] = a.p_ref;
                if constexpr (NV == 5) W[4] = bw;
            } else {
                W = c2p(a.eos, read_cell<NV>(a.U, a.m.plane, cell));
                W[1] = bu;
                W[2] = bvv;
                if constexpr (NV == 5) W[4] = bw;
            }
            out = p2c(a.eos, W);
        }
        if (a.reset) {
#pragma unroll
            for (int v = 0; v < NV; ++v) a.Uout[v * a.m.plane + cell] = out[v];
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) a.forced[5 * (long long)k + v] = out[v];
        }
    }
}

// ImmersedBoundary::fill_fresh (Physics.cpp:1336-1354): the cells a moving body left take the image-point state with the
// velocity relative to the wall scaled by the ratio of the distances; the probes read settled cells only, so in place.
struct FreshArgs {
    Mesh m;
    Eos<double> eos;
    int n;
    const int* cell;          // [n]
    const int* img_cell;      // [8 n]
    const double* img_w;      // [8 n]
    const double* ratio;      // [n]
    const double* wvel;       // [3 n]
    double* U;
};

template <int NV> __global__ void fresh_fill_kernel(const FreshArgs a) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n; k += gridDim.x * blockDim.x) {
        double W[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int q = 0; q < 8; ++q) {
            const double w = a.img_w[8 * k + q];
            if (w == 0.0) continue;
            const St<double, NV> Wq = c2p(a.eos, read_cell<NV>(a.U, a.m.plane, a.img_cell[8 * k + q]));
#pragma unroll
            for (int v = 0; v < NV; ++v) W[v] += w * Wq[v];
        }
        const double r = a.ratio[k], wu = a.wvel[3 * k], wv = a.wvel[3 * k + 1], ww = a.wvel[3 * k + 2];
        St<double, NV> Wf;
        Wf[0] = W[0];
        Wf[1] = wu + r * (W[1] - wu);
        Wf[2] = wv + r * (W[2] - wv);
        Wf[3] = W[3];
        if constexpr (NV == 5) Wf[4] = ww + r * (W[4] - ww);
        const St<double, NV> out = p2c(a.eos, Wf);
        const long long c = a.cell[k];
#pragma unroll
        for (int v = 0; v < NV; ++v) a.U[v * a.m.plane + c] = out[v];
    }
}

}   // namespace fvg
