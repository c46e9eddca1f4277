// Navier-Stokes viscous and heat fluxes on a 3-D mesh (NavierStokes::viscous_residual_3d, cpp/src/Physics.cpp:484-830).
//
// A CTA owns a TX x TY x TZ tile. It first stages the reference's padded conservative state of the tile and one cell
// around it in shared memory (padded_3d + fix_padded_corners semantics, a periodic side wrapped), then sweeps its axes
// in turn, like the stage kernel. Per axis d:
//   1. cells:   for the tile extended by one cell along d, the four velocity-gradient entries
//               G[a][b] = (d(rho u_a)/dx_b - u_a d(rho)/dx_b) / rho that the faces of axis d read (central differences of
//               the padded conservative state);
//   2. faces:   velocity and T = p / rho on both sides, compact normal derivatives, face-averaged cross derivatives,
//               Stokes stress and Fourier heat flux;
//   3. balance: ((0 + (Fr - Fl)) + (Ft - Fb)) + (Fk - Ff), accumulated in shared memory in that order.
// The result, times 1 / volume, is the viscous residual Rv of every cell (added to the inviscid one by the stage
// kernel, R + Rv being the reference's `r += ...`), and each CTA writes the largest viscous speed bound of its cells
// (ViscousBound.hpp: max |u_a| + c + 2 L sum(1/h^2) max(4/3 mu/rho, k (gamma-1)/rho) + 1e-12).
#pragma once

#include <type_traits>

#include "grid.cuh"

namespace fvg {

struct ViscArgs {
    Mesh m;
    Bc bc;
    Eos<double> eos;
    double mu, k_cond, L, inv_h2;
    double u_in, v_in;
    int bface2;        // boundary_order == 2
    int periodic[3];   // both sides of the axis periodic
    int through[6];    // the side is periodic or a part interface (kHaloPeer): no wall rules at its faces
    int nvar;          // state planes: 4 on a 2-D mesh (rho w is +0 there), 5 in 3-D
    const double* U;
    double* Rv;
    float* Rvf;        // the 3-D mixed form: the FP32 viscous balance sums of the planes 1 .. 4 (StageArgs::Rvf)
    double* blockmax;
    const int* gate;   // the kernel does nothing unless *gate
    int tiles[3];
    int b0;            // the tile of the launch's first CTA (a launch over a range of tiles; 0: all)
};

// the zero-gradient copy with the momentum rules of a wall side (BoundaryManager::viscous_ghost_3d, Boundaries.cpp:258-275)
__device__ __forceinline__ St<double, 5> viscous_ghost_3d(const ViscArgs& a, int side, const St<double, 5>& c) {
    St<double, 5> gh = c;
    const int d = side >> 1;
    const int type = a.bc.type[side];
    const int mom[3] = {1, 2, 4};
    if (type == kBcNoSlip) {
        gh[1] = -c[1];
        gh[2] = -c[2];
        gh[4] = -c[4];
    } else if (type == kBcWall) {
        gh[mom[d]] = -c[mom[d]];
    } else if (type == kBcMovingWall) {
        const double uw[3] = {a.bc.tv ? a.bc.tv[0] : a.u_in, a.bc.tv ? a.bc.tv[1] : a.v_in, 0.0};
#pragma unroll
        for (int t = 0; t < 3; ++t) gh[mom[t]] = (t == d) ? -c[mom[t]] : 2.0 * c[0] * uw[t] - c[mom[t]];
        if (a.bface2)   // match_kinetic_energy (Boundaries.cpp:197-200)
            gh[3] = c[3] + 0.5 * (gh[1] * gh[1] + gh[2] * gh[2] + gh[4] * gh[4] - c[1] * c[1] - c[2] * c[2] - c[4] * c[4]) / c[0];
    }
    return gh;
}

__device__ __forceinline__ St<double, 5> cell_at(const ViscArgs& a, int i, int j, int k) {
    const long long c = ((long long)k * a.m.ny + j) * a.m.nx + i;
    if (a.nvar == 5) return read_state<5>(a.bc, a.U, a.m.plane, c);
    const St<double, 4> u4 = read_state<4>(a.bc, a.U, a.m.plane, c);
    St<double, 5> u;
#pragma unroll
    for (int s = 0; s < 4; ++s) u[s] = u4[s];
    u[4] = 0.0;
    return u;
}

// The padded entry beyond one side along axis d (padded_3d, Boundaries.cpp:621-700): the opposite layer of a periodic
// side, the wall ghost of a wall side, else the replicated edge cell. idx[d] is -1 or n_d; the other indices are inside.
__device__ __forceinline__ St<double, 5> face_ghost(const ViscArgs& a, int d, int idx0, int idx1, int idx2) {
    int idx[3] = {idx0, idx1, idx2};
    const int n3[3] = {a.m.nx, a.m.ny, a.m.nz};
    const bool hi = idx[d] >= n3[d];
    const int side = 2 * d + (hi ? 1 : 0);
    const int type = a.bc.type[side];
    if (type == kBcPeriodic) {
        idx[d] = hi ? 0 : n3[d] - 1;
        return cell_at(a, idx[0], idx[1], idx[2]);
    }
    idx[d] = hi ? n3[d] - 1 : 0;
    const St<double, 5> c = cell_at(a, idx[0], idx[1], idx[2]);
    if (type == kBcNoSlip || type == kBcWall || type == kBcMovingWall) return viscous_ghost_3d(a, side, c);
    return c;
}

// Any entry of the reference's padded conservative state, cell indices -1 .. n per axis: the cell, a face ghost, an
// edge (two axes outside: fix_padded_corners, Boundaries.cpp:509-548, with boundary_order = 2, else edge replication)
// or a corner (replication).
__device__ __forceinline__ St<double, 5> padded_cons(const ViscArgs& a, int i, int j, int k) {
    const int n3[3] = {a.m.nx, a.m.ny, a.m.nz};
    int p[3] = {i, j, k};
    int ng = 0, ga[2] = {-1, -1};
#pragma unroll
    for (int d = 0; d < 3; ++d)
        if (!held(a.bc, d, p[d], n3[d])) {
            if (ng < 2) ga[ng] = d;
            ++ng;
        }
    if (ng == 0) return cell_at(a, i, j, k);
    if (ng == 1) return face_ghost(a, ga[0], i, j, k);
    if (ng == 2 && a.bface2) {
        const int d = ga[0], e = ga[1];
        const bool hi = p[d] >= n3[d];
        int q[3] = {p[0], p[1], p[2]};
        q[d] = hi ? n3[d] - 1 : 0;
        const int side = 2 * d + (hi ? 1 : 0);
        if (a.bc.type[side] == kBcPeriodic) {
            q[d] = hi ? 0 : n3[d] - 1;
            return face_ghost(a, e, q[0], q[1], q[2]);
        }
        return viscous_ghost_3d(a, side, face_ghost(a, e, q[0], q[1], q[2]));
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int lo = -a.bc.ext[2 * d], hi = n3[d] - 1 + a.bc.ext[2 * d + 1];
        p[d] = p[d] < lo ? lo : (p[d] > hi ? hi : p[d]);
    }
    return cell_at(a, p[0], p[1], p[2]);
}

// The range of positions a viscous box loads along an axis: one ghost layer beyond a side, or the neighbouring part's
// ghost planes beyond a part interface.
__device__ __forceinline__ int box_clamp(const ViscArgs& a, int d, int g, int n) {
    const int lo = a.bc.ext[2 * d] > 0 ? -a.bc.ext[2 * d] : -1, hi = a.bc.ext[2 * d + 1] > 0 ? n - 1 + a.bc.ext[2 * d + 1] : n;
    return g < lo ? lo : (g > hi ? hi : g);
}

// velocity component a (0, 1, 2) of a primitive state, without indexing the state by a run-time value
__device__ __forceinline__ double velc(const St<double, 5>& w, int a) { return a == 0 ? w[1] : (a == 1 ? w[2] : w[4]); }

template <int TX, int TY, int TZ> struct ViscShape {
    static constexpr int NC = TX * TY * TZ;
    static constexpr int BX = TX + 2, BY = TY + 2, BZ = TZ + 2, NB = BX * BY * BZ;   // padded box of the tile
    static constexpr int cmax(int x, int y) { return x > y ? x : y; }
    static constexpr int NE = cmax(cmax((TX + 2) * TY * TZ, TX * (TY + 2) * TZ), TX * TY * (TZ + 2));
    static constexpr int NF = cmax(cmax((TX + 1) * TY * TZ, TX * (TY + 1) * TZ), TX * TY * (TZ + 1));
    // B [5][NB] padded conservative box, G [4][NE] gradient entries, F [4][NF] face fluxes (components 1..4), acc [5][NC], red [32]
    static constexpr int SMEM_DOUBLES = 5 * NB + 4 * NE + 4 * NF + 5 * NC + 32;
    static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

template <int TX, int TY, int TZ, int NT>
__global__ void __launch_bounds__(NT) viscous_kernel(const ViscArgs a) {
    using S = ViscShape<TX, TY, TZ>;
    constexpr int NC = S::NC, BX = S::BX, BY = S::BY, NB = S::NB;
    extern __shared__ double smem[];
    double* B = smem;                 // [5][NB]
    double* G = B + 5 * NB;           // [4][NE]
    double* Fv = G + 4 * S::NE;       // [4][NF]
    double* acc = Fv + 4 * S::NF;     // [5][NC]
    double* red = acc + 5 * NC;
    if (!*a.gate) return;
    const Mesh& m = a.m;
    const int tid = threadIdx.x, b = blockIdx.x + a.b0;
    const int o3[3] = {(b % a.tiles[0]) * TX, ((b / a.tiles[0]) % a.tiles[1]) * TY, (b / (a.tiles[0] * a.tiles[1])) * TZ};
    const int n3[3] = {m.nx, m.ny, m.nz};
    const double h[3] = {m.dx, m.dy, m.dz};
    // the momentum slots of the velocity components, and the (a, b) of the four gradient entries the faces of axis d read,
    // in the reference's CrossGhosts order (cpp/src/Physics.cpp:653-667); compile-time tables, constant indices in the
    // unrolled sweeps
    constexpr int mom[3] = {1, 2, 4};
    constexpr int GA[3][4] = {{0, 1, 2, 0}, {0, 1, 2, 1}, {0, 1, 2, 2}};
    constexpr int GB[3][4] = {{1, 1, 2, 2}, {0, 0, 2, 2}, {0, 1, 0, 1}};
    // box position (tile-relative cell index -1 .. T per axis) -> shared-memory index
    auto bidx = [&](int i, int j, int k) { return ((k + 1) * BY + (j + 1)) * BX + (i + 1); };
    auto cons = [&](int p) {
        St<double, 5> u;
#pragma unroll
        for (int q = 0; q < 5; ++q) u[q] = B[q * NB + p];
        return u;
    };

    // whether a side of the tile lies on a side of the mesh that is neither periodic nor a part interface (without one,
    // every box position is a cell the arrays hold, after the periodic wrap, and no face of the tile has a wall rule),
    // and whether the tile lies wholly inside the mesh
    bool walls = false;
#pragma unroll
    for (int x = 0; x < 3; ++x)
        walls = walls || (o3[x] == 0 && !a.through[2 * x]) || (o3[x] + (x == 0 ? TX : (x == 1 ? TY : TZ)) >= n3[x] && !a.through[2 * x + 1]);
    const bool full = o3[0] + TX <= n3[0] && o3[1] + TY <= n3[1] && o3[2] + TZ <= n3[2];

    // ---- 0. the padded conservative state of the tile and one cell around it. A position beyond a periodic side is the
    // wrapped cell (so the box holds the neighbours the reference reads for that cell); the rest is the reference's
    // padded array (padded_cons). The eight corners are never read.
    for (int e = tid; e < NB; e += NT) {
        int g[3] = {o3[0] + e % BX - 1, o3[1] + (e / BX) % BY - 1, o3[2] + e / (BX * BY) - 1};
#pragma unroll
        for (int x = 0; x < 3; ++x)
            if (a.periodic[x] && (g[x] < 0 || g[x] >= n3[x])) g[x] = ((g[x] % n3[x]) + n3[x]) % n3[x];
        // a tile that overhangs the mesh: positions past the ghost layer are clamped onto it (their results are not used)
#pragma unroll
        for (int x = 0; x < 3; ++x) g[x] = box_clamp(a, x, g[x], n3[x]);
        const St<double, 5> u = walls ? padded_cons(a, g[0], g[1], g[2]) : cell_at(a, g[0], g[1], g[2]);
#pragma unroll
        for (int q = 0; q < 5; ++q) B[q * NB + e] = u[q];
    }
    __syncthreads();

// one sweep per axis, the axis a compile-time constant (every small index array stays in registers)
    auto sweep = [&](auto axis_c) {
        constexpr int d = decltype(axis_c)::value;
        constexpr int E[3] = {TX + (d == 0 ? 2 : 0), TY + (d == 1 ? 2 : 0), TZ + (d == 2 ? 2 : 0)};
        constexpr int Fd[3] = {TX + (d == 0), TY + (d == 1), TZ + (d == 2)};
        const int nE = E[0] * E[1] * E[2], nF = Fd[0] * Fd[1] * Fd[2];
        // ---- 1. the four gradient entries of the cells of the tile extended along d (meaningless at a ghost position)
        for (int e = tid; e < nE; e += NT) {
            int l[3] = {e % E[0], (e / E[0]) % E[1], e / (E[0] * E[1])};
            l[d] -= 1;
            const int p = bidx(l[0], l[1], l[2]);
            const St<double, 5> w = c2p(a.eos, cons(p));
            const double rho = w[0];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int ga = GA[d][s], gb = GB[d][s];
                const int off = gb == 0 ? 1 : (gb == 1 ? BX : BX * BY);
                const double gq = (B[mom[ga] * NB + p + off] - B[mom[ga] * NB + p - off]) / (2.0 * h[gb]);
                const double g0 = (B[p + off] - B[p - off]) / (2.0 * h[gb]);
                G[s * S::NE + e] = (gq - velc(w, ga) * g0) / rho;
            }
        }
        __syncthreads();
        // ---- 2. faces
        const double area = m.area[d];
        const int estride = d == 0 ? 1 : (d == 1 ? E[0] : E[0] * E[1]);
        const int bstride = d == 0 ? 1 : (d == 1 ? BX : BX * BY);
        for (int f = tid; f < nF; f += NT) {
            const int f3[3] = {f % Fd[0], (f / Fd[0]) % Fd[1], f / (Fd[0] * Fd[1])};
            const int g3[3] = {o3[0] + f3[0], o3[1] + f3[1], o3[2] + f3[2]};
            const int t = g3[d];
            bool inside = true;
            if (!full)
#pragma unroll
                for (int x = 0; x < 3; ++x) inside = inside && (x == d ? g3[x] <= n3[x] : g3[x] < n3[x]);
            double out[4] = {0.0, 0.0, 0.0, 0.0};
            if (inside) {
                const bool lo = walls && t == 0, hi = walls && t == n3[d];
                const int eL = (f3[2] * E[1] + f3[1]) * E[0] + f3[0];   // extended position of the cell t-1 (or the ghost)
                const int eR = eL + estride;
                int lc[3] = {f3[0], f3[1], f3[2]};
                lc[d] -= 1;
                const int pL = bidx(lc[0], lc[1], lc[2]), pR = pL + bstride;
                const St<double, 5> wL = c2p(a.eos, cons(pL)), wR = c2p(a.eos, cons(pR));
                const double vL[3] = {wL[1], wL[2], wL[4]}, vR[3] = {wR[1], wR[2], wR[4]};
                const double TL = wL[3] / wL[0], TR = wR[3] / wR[0];
                // cross terms: the cells on either side; at a side that is not periodic the cell next to it (both slots)
                const bool lo_wall = lo && !a.through[2 * d], hi_wall = hi && !a.through[2 * d + 1];
                const int xL = lo_wall ? eR : eL;
                const int xR = hi_wall ? eL : eR;
                const bool phys = a.bface2 && (lo_wall || hi_wall);
                double Gc[4];
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    if (phys) {
                        // d u_a / d x_b from the tangential difference of the face values (ghost and cell averages)
                        const int ga = GA[d][s], gb = GB[d][s];
                        const int pg = lo ? pL : pR, pc = lo ? pR : pL;
                        const int off = gb == 0 ? 1 : (gb == 1 ? BX : BX * BY);
                        double fc[2];
#pragma unroll
                        for (int w2 = 0; w2 < 2; ++w2) {
                            const int o = w2 == 0 ? off : -off;
                            const St<double, 5> wg = c2p(a.eos, cons(pg + o));
                            const St<double, 5> wc = c2p(a.eos, cons(pc + o));
                            fc[w2] = 0.5 * (velc(wg, ga) + velc(wc, ga));
                        }
                        Gc[s] = (fc[0] - fc[1]) / (2.0 * h[gb]);
                    } else {
                        Gc[s] = 0.5 * (G[s * S::NE + xL] + G[s * S::NE + xR]);
                    }
                }
                double Gn[3], vf[3];
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    Gn[x] = (vR[x] - vL[x]) / h[d];
                    vf[x] = 0.5 * (vL[x] + vR[x]);
                }
                const double dT = (TR - TL) / h[d];
                // Gc slots: d=0: [du/dy, dv/dy, dw/dz, du/dz]; d=1: [du/dx, dv/dx, dw/dz, dv/dz]; d=2: [du/dx, dv/dy, dw/dx, dw/dy]
                double tau[3];
                if (d == 0) {
                    tau[0] = a.mu * ((4.0 / 3.0) * Gn[0] - (2.0 / 3.0) * ((0.0 + Gc[1]) + Gc[2]));
                    tau[1] = a.mu * (Gn[1] + Gc[0]);
                    tau[2] = a.mu * (Gn[2] + Gc[3]);
                } else if (d == 1) {
                    tau[0] = a.mu * (Gn[0] + Gc[1]);
                    tau[1] = a.mu * ((4.0 / 3.0) * Gn[1] - (2.0 / 3.0) * ((0.0 + Gc[0]) + Gc[2]));
                    tau[2] = a.mu * (Gn[2] + Gc[3]);
                } else {
                    tau[0] = a.mu * (Gn[0] + Gc[2]);
                    tau[1] = a.mu * (Gn[1] + Gc[3]);
                    tau[2] = a.mu * ((4.0 / 3.0) * Gn[2] - (2.0 / 3.0) * ((0.0 + Gc[0]) + Gc[1]));
                }
                const double q_d = -a.k_cond * dT;
                out[0] = tau[0] * area;
                out[1] = tau[1] * area;
                out[2] = (vf[0] * tau[0] + vf[1] * tau[1] + vf[2] * tau[2] - q_d) * area;
                out[3] = tau[2] * area;
            }
#pragma unroll
            for (int x = 0; x < 4; ++x) Fv[x * S::NF + f] = out[x];
        }
        __syncthreads();
        // ---- 3. balance (component 0 of every viscous flux is +0)
        for (int c = tid; c < NC; c += NT) {
            const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
            const int fl = (c3[2] * Fd[1] + c3[1]) * Fd[0] + c3[0];
            const int fr = fl + (d == 0 ? 1 : (d == 1 ? Fd[0] : Fd[0] * Fd[1]));
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double dif = q == 0 ? 0.0 - 0.0 : Fv[(q - 1) * S::NF + fr] - Fv[(q - 1) * S::NF + fl];
                acc[q * NC + c] = d == 0 ? 0.0 + dif : acc[q * NC + c] + dif;
            }
        }
        // (no barrier: each thread balances its own cells, the same ones in every sweep and in the epilogue, and the
        // next sweep's gradients touch neither Fv nor acc; its faces come after its own barrier)
    };
    sweep(std::integral_constant<int, 0>{});
    sweep(std::integral_constant<int, 1>{});
    sweep(std::integral_constant<int, 2>{});
    // ---- residual and speed bound
    double smax = 0.0;
    for (int c = tid; c < NC; c += NT) {
        const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
        const int g3[3] = {o3[0] + c3[0], o3[1] + c3[1], o3[2] + c3[2]};
        if (g3[0] >= m.nx || g3[1] >= m.ny || g3[2] >= m.nz) continue;
        const long long cell = ((long long)g3[2] * m.ny + g3[1]) * m.nx + g3[0];
#pragma unroll
        for (int q = 0; q < 5; ++q) a.Rv[q * m.plane + cell] = acc[q * NC + c] * m.inv_cell;
        const St<double, 5> w = c2p(a.eos, cons(bidx(c3[0], c3[1], c3[2])));
        const double rho = w[0];
        const double nu_eff = vmax((4.0 / 3.0) * (a.mu / rho), (a.k_cond * (a.eos.gamma - 1.0)) / rho) + 1e-12;
        const double vm = vmax(vmax(fabs(w[1]), fabs(w[2])), fabs(w[4]));
        const double s = vm + sound_speed(a.eos, w[3], rho) + 2.0 * a.L * a.inv_h2 * nu_eff;
        if (s > smax) smax = s;
    }
    const double bm = block_max<NT>(smax, red);
    if (tid == 0) a.blockmax[b] = bm;
}

}   // namespace fvg

namespace fvg {

// ---------------------------------------------------------------------------------------------- 2-D viscous sweep
// NavierStokes::viscous_residual_rows (cpp/src/Physics.cpp:229-479) on a TX x TY tile: the padded frame of the 2-D mesh
// (get_padded_frame + fix_frame_corners, cpp/src/Boundaries.cpp:402-630: the zero-gradient copy with the wall momentum
// rules, the same entries padded_cons gives a one-cell-high 3-D mesh; a periodic side wrapped) staged for the tile and
// two cells around it; then, for the tile and one cell around it, the cell quantities of a row (u, v, T and the four
// velocity derivatives (d(rho u_a)/dx_b - u_a d(rho)/dx_b) / rho from central differences over 2h); then the x and y face
// fluxes with the reference's choice of cells at the mesh sides (a side that is not periodic averages the derivative of
// the boundary cell with itself, or, with boundary_order 2, takes the tangential derivative of the face-averaged frame);
// then the balance ((0 + (Fr - Fl)) + (Ft - Fb)) / area and the speed bound max(|u|, |v|) + c + 2 L (1/dx^2 + 1/dy^2) nu_eff.
template <int TX, int TY> struct Visc2Shape {
    static constexpr int BX = TX + 4, BY = TY + 4, NB = BX * BY;   // conservative box: the tile +- 2
    static constexpr int QX = TX + 2, QY = TY + 2, NQ = QX * QY;   // cell quantities: the tile +- 1
    static constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1);
    // doubles: B [4][NB], Q [7][NQ] (u, v, T, du/dx, du/dy, dv/dx, dv/dy), FX [3][NFX], FY [3][NFY], 32 for the reduction
    static constexpr int SMEM_DOUBLES = 4 * NB + 7 * NQ + 3 * NFX + 3 * NFY + 32;
    static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) viscous2d_kernel(const ViscArgs a) {
    using S = Visc2Shape<TX, TY>;
    constexpr int BX = S::BX, NB = S::NB, QX = S::QX, NQ = S::NQ;
    constexpr double MU_DIAG = 4.0 / 3.0, MU_OFF = 2.0 / 3.0;
    extern __shared__ double smem[];
    double* B = smem;                 // [4][NB]
    double* Q = B + 4 * NB;           // [7][NQ]
    double* FX = Q + 7 * NQ;          // [3][NFX]
    double* FY = FX + 3 * S::NFX;     // [3][NFY]
    double* red = FY + 3 * S::NFY;
    if (!*a.gate) return;
    const Mesh& m = a.m;
    const int tid = threadIdx.x, b = blockIdx.x + a.b0;
    const int ox = (b % a.tiles[0]) * TX, oy = (b / a.tiles[0]) * TY;
    const int nx = m.nx, ny = m.ny;
    const double dx = m.dx, dy = m.dy, mu = a.mu, kc = a.k_cond;
    const bool px = a.periodic[0] != 0, py = a.periodic[1] != 0;
    // box position (tile-relative -2 .. T+1) and quantity position (-1 .. T)
    auto bidx = [&](int i, int j) { return (j + 2) * BX + (i + 2); };
    auto qidx = [&](int i, int j) { return (j + 1) * QX + (i + 1); };
    auto q = [&](int s, int i, int j) { return Q[s * NQ + qidx(i, j)]; };

    // ---- the padded state of the tile +- 2 (the frame beyond the mesh, a periodic side wrapped first)
    for (int e = tid; e < NB; e += NT) {
        int g[2] = {ox + e % BX - 2, oy + e / BX - 2};
        if (px && (g[0] < 0 || g[0] >= nx)) g[0] = ((g[0] % nx) + nx) % nx;
        if (py && (g[1] < 0 || g[1] >= ny)) g[1] = ((g[1] % ny) + ny) % ny;
        g[0] = box_clamp(a, 0, g[0], nx);
        g[1] = box_clamp(a, 1, g[1], ny);
        const St<double, 5> u = padded_cons(a, g[0], g[1], 0);
#pragma unroll
        for (int s = 0; s < 4; ++s) B[s * NB + e] = u[s];
    }
    __syncthreads();
    // ---- cell quantities of the tile +- 1 (the expressions of fill / scalar_cells)
    for (int e = tid; e < NQ; e += NT) {
        const int i = e % QX - 1, j = e / QX - 1;
        const int p = bidx(i, j);
        St<double, 5> c;
#pragma unroll
        for (int s = 0; s < 4; ++s) c[s] = B[s * NB + p];
        c[4] = 0.0;
        const St<double, 5> w = c2p(a.eos, c);
        const double rho = w[0], u = w[1], v = w[2];
        const int pe = p + 1, pw = p - 1, pn = p + BX, ps = p - BX;
        const double drx = (B[pe] - B[pw]) / (2.0 * dx), dry = (B[pn] - B[ps]) / (2.0 * dy);
        const double gx1 = (B[NB + pe] - B[NB + pw]) / (2.0 * dx), gy1 = (B[NB + pn] - B[NB + ps]) / (2.0 * dy);
        const double gx2 = (B[2 * NB + pe] - B[2 * NB + pw]) / (2.0 * dx), gy2 = (B[2 * NB + pn] - B[2 * NB + ps]) / (2.0 * dy);
        Q[0 * NQ + e] = u;
        Q[1 * NQ + e] = v;
        Q[2 * NQ + e] = w[3] / rho;
        Q[3 * NQ + e] = (gx1 - u * drx) / rho;
        Q[4 * NQ + e] = (gy1 - u * dry) / rho;
        Q[5 * NQ + e] = (gx2 - v * drx) / rho;
        Q[6 * NQ + e] = (gy2 - v * dry) / rho;
    }
    __syncthreads();
    // ---- x faces of the tile's rows (xflux): face il between quantity positions il-1 and il
    for (int f = tid; f < S::NFX; f += NT) {
        const int il = f % (TX + 1), jl = f / (TX + 1);
        const int i = ox + il, j = oy + jl;
        double out[3] = {0.0, 0.0, 0.0};
        if (i <= nx && j < ny) {
            const bool lo = i == 0, hi = i == nx;
            const double uL = q(0, il - 1, jl), uR = q(0, il, jl);
            const double vL = q(1, il - 1, jl), vR = q(1, il, jl);
            const double TL = q(2, il - 1, jl), TR = q(2, il, jl);
            const double u_f = 0.5 * (uL + uR), v_f = 0.5 * (vL + vR);
            const double du_dx = (uR - uL) / dx, dv_dx = (vR - vL) / dx, dT_dx = (TR - TL) / dx;
            // the cells whose tangential derivatives the face averages: the two neighbours; at a side that is not
            // periodic, the boundary cell twice
            const bool lo_wall = lo && !a.through[0], hi_wall = hi && !a.through[1];
            const int xl = lo_wall ? il : il - 1, xr = hi_wall ? il - 1 : il;
            double du_dy = 0.5 * (q(4, xl, jl) + q(4, xr, jl));
            double dv_dy = 0.5 * (q(6, xl, jl) + q(6, xr, jl));
            if (a.bface2 && (lo_wall || hi_wall)) {
                const int ig = lo ? il - 1 : il, ic = lo ? il : il - 1;   // the frame column and the boundary cell's column
                const double fu_p = 0.5 * (q(0, ig, jl + 1) + q(0, ic, jl + 1)), fu_m = 0.5 * (q(0, ig, jl - 1) + q(0, ic, jl - 1));
                const double fv_p = 0.5 * (q(1, ig, jl + 1) + q(1, ic, jl + 1)), fv_m = 0.5 * (q(1, ig, jl - 1) + q(1, ic, jl - 1));
                du_dy = (fu_p - fu_m) / (2.0 * dy);
                dv_dy = (fv_p - fv_m) / (2.0 * dy);
            }
            const double tau_xx = mu * (MU_DIAG * du_dx - MU_OFF * dv_dy);
            const double tau_xy = mu * (du_dy + dv_dx);
            const double q_x = -kc * dT_dx;
            out[0] = tau_xx * dy;
            out[1] = tau_xy * dy;
            out[2] = (u_f * tau_xx + v_f * tau_xy - q_x) * dy;
        }
#pragma unroll
        for (int s = 0; s < 3; ++s) FX[s * S::NFX + f] = out[s];
    }
    // ---- y faces of the tile's columns (yflux): face jl between quantity rows jl-1 and jl
    for (int f = tid; f < S::NFY; f += NT) {
        const int il = f % TX, jl = f / TX;
        const int i = ox + il, j = oy + jl;
        double out[3] = {0.0, 0.0, 0.0};
        if (i < nx && j <= ny) {
            const bool lo = j == 0, hi = j == ny;
            const double uB = q(0, il, jl - 1), uT = q(0, il, jl);
            const double vB = q(1, il, jl - 1), vT = q(1, il, jl);
            const double TB = q(2, il, jl - 1), TT = q(2, il, jl);
            const double u_f = 0.5 * (uB + uT), v_f = 0.5 * (vB + vT);
            const double dv_dy = (vT - vB) / dy, du_dy = (uT - uB) / dy, dT_dy = (TT - TB) / dy;
            const bool lo_wall = lo && !a.through[2], hi_wall = hi && !a.through[3];
            const int yb = lo_wall ? jl : jl - 1, yt = hi_wall ? jl - 1 : jl;
            double du_dx = 0.5 * (q(3, il, yb) + q(3, il, yt));
            double dv_dx = 0.5 * (q(5, il, yb) + q(5, il, yt));
            if (a.bface2 && (lo_wall || hi_wall)) {
                const int jg = lo ? jl - 1 : jl, jc = lo ? jl : jl - 1;   // the frame row and the boundary cell's row
                const double fu_p = 0.5 * (q(0, il + 1, jg) + q(0, il + 1, jc)), fu_m = 0.5 * (q(0, il - 1, jg) + q(0, il - 1, jc));
                const double fv_p = 0.5 * (q(1, il + 1, jg) + q(1, il + 1, jc)), fv_m = 0.5 * (q(1, il - 1, jg) + q(1, il - 1, jc));
                du_dx = (fu_p - fu_m) / (2.0 * dx);
                dv_dx = (fv_p - fv_m) / (2.0 * dx);
            }
            const double tau_yy = mu * (MU_DIAG * dv_dy - MU_OFF * du_dx);
            const double tau_yx = mu * (du_dy + dv_dx);
            const double q_y = -kc * dT_dy;
            out[0] = tau_yx * dx;
            out[1] = tau_yy * dx;
            out[2] = (u_f * tau_yx + v_f * tau_yy - q_y) * dx;
        }
#pragma unroll
        for (int s = 0; s < 3; ++s) FY[s * S::NFY + f] = out[s];
    }
    __syncthreads();
    // ---- balance, residual and speed bound
    const double inv_area = m.inv_cell;
    const double zero_slot = ((0.0 + (0.0 - 0.0)) + (0.0 - 0.0)) * inv_area;
    double smax = 0.0;
    for (int c = tid; c < TX * TY; c += NT) {
        const int il = c % TX, jl = c / TX;
        const int i = ox + il, j = oy + jl;
        if (i >= nx || j >= ny) continue;
        const long long cell = (long long)j * nx + i;
        const int fl = jl * (TX + 1) + il, fb = jl * TX + il;
        a.Rv[cell] = zero_slot;
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const double bal = ((0.0 + (FX[s * S::NFX + fl + 1] - FX[s * S::NFX + fl])) + (FY[s * S::NFY + fb + TX] - FY[s * S::NFY + fb])) * inv_area;
            a.Rv[(s + 1) * m.plane + cell] = bal;
        }
        St<double, 5> cc;
#pragma unroll
        for (int s = 0; s < 4; ++s) cc[s] = B[s * NB + bidx(il, jl)];
        cc[4] = 0.0;
        const St<double, 5> w = c2p(a.eos, cc);
        const double rho = w[0];
        const double nu_eff = vmax((4.0 / 3.0) * (a.mu / rho), (a.k_cond * (a.eos.gamma - 1.0)) / rho) + 1e-12;
        const double s = vmax(fabs(w[1]), fabs(w[2])) + sound_speed(a.eos, w[3], rho) + 2.0 * a.L * a.inv_h2 * nu_eff;
        if (s > smax) smax = s;
    }
    const double bm = block_max<NT>(smax, red);
    if (tid == 0) a.blockmax[b] = bm;
}

}   // namespace fvg
