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
            // in 2-D the reference's velocity index 4 is the z component, here the last of 4 is the pressure
            const double wz = NV == 5 ? W[4] : 0.0;
            const double un = NV == 5 ? W[1] * nx + W[2] * ny + wz * nz : W[1] * nx + W[2] * ny;
            double ux, uy, uz = 0.0;
            if (a.slip) {   // tangential velocity kept, normal velocity reflected through zero at the wall
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
            St<double, NV> W;
            if (a.reset) {
                W[0] = a.rho_ref;
                W[1] = 0.0;
                W[2] = 0.0;
                W[3] = a.p_ref;
                if constexpr (NV == 5) W[4] = 0.0;
            } else {
                W = c2p(a.eos, read_cell<NV>(a.U, a.m.plane, cell));
                W[1] = 0.0;
                W[2] = 0.0;
                if constexpr (NV == 5) W[4] = 0.0;
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

}   // namespace fvg
