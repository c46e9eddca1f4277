// The cell engine of an adaptive mesh on the device, for meshes whose leaves are all of level 0: the reference's
// CellFluxEngine (cpp/include/fv/CellFlux.hpp; stencils built once per mesh in cpp/src/CellFlux.cpp, one flux per face
// and the cells' gather in cpp/src/CellFluxResidual.cpp) and CellAdvance (cpp/include/fv/CellAdvance.hpp) with one level.
//
// The mesh is a list of leaves in the caller's order (the reference keeps them sorted by level and Morton key, so
// neighbours along every axis sit close together in the arrays). The state lives in HBM as planes over the leaves
// (plane q of leaf c at q * lplane + c). The engine is three kernels per residual:
//   k_cells_prim    the primitive state of every leaf once (the reference's prepare / refresh_all);
//   k_cells_faces   one thread per face: its stencil gathered through an index table (six entries with WENO5-Z, four
//                   with MUSCL / WENO3-Z), each entry a leaf's primitive state or a ghost layer of a physical side (the
//                   side's ghost_state of a leaf, then cons_to_prim), the two face states, the Riemann solver, the flux
//                   and the face's wave speed (CellFluxEngine::fluxes, CellFluxResidual.cpp:21-358);
//   k_cells_gather  one thread per leaf: the flux of each side times the face's measure, summed in the reference's order
//                   (((0 - (G1 - G0)) - (G3 - G2)) - (G5 - G4)) / volume (CellFluxEngine::gather, CellFluxResidual.cpp:974-1086),
//                   fused with the stage update of the time scheme (R, U + dt R, or a U0 + b (U + dt R)).
// The stencil table is what the reference's build makes for level-0 leaves (beyond / face_stencil / far_code,
// CellFlux.cpp:444-560): a side of a leaf on a physical edge replicates the leaf, a periodic axis wraps; with
// boundary_order = 2 an entry that replicates a leaf at a wall, inlet or outlet becomes that side's ghost layer of the
// mirrored leaf, and the boundary faces are reconstructed through three (WENO5-Z) or two ghost layers. With level-0
// leaves only the residual has the bits of the uniform solver's, as the reference's own tests check for its engine.
#include "../../include/fenice_gpu.h"
#include "host_common.h"
#include "hancock.cuh"
#include "stage.cuh"
#include "viscous.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

struct fvg_cells {
    fvg_config cfg{};
    int dim = 3, nvar = 5, ns = 6;
    long long nleaf = 0, lplane = 0, nface = 0, fplane = 0;
    fvg::Eos<double> eos{};
    fvg::Bc bc{};
    double length[3] = {0, 0, 0};   // the measure of a face normal to each axis (Mesh::face_area)
    double inv_vol = 0.0;           // 1 / the volume (area in 2-D) of a leaf
    cudaStream_t stream = nullptr;
    double *U = nullptr, *Ut = nullptr, *W = nullptr, *R = nullptr, *F = nullptr, *staging = nullptr;
    int *code = nullptr, *meta = nullptr, *side_face = nullptr;
    // the viscous terms (3-D): the neighbour table, the cell quantities and the viscous face fluxes
    bool visc = false;
    int* nbr = nullptr;
    double *Q = nullptr, *Fv = nullptr;   // Q: 13 planes in 3-D, 7 in 2-D
    double mu = 0.0, k_cond = 0.0, L = 0.0, inv_h2 = 0.0, h[3] = {0, 0, 0};
    double *PL = nullptr, *PR = nullptr;  // MUSCL-Hancock: the face states of the faces' two sides
    unsigned long long* smax = nullptr;   // [3]: the bits of the largest face speed of each stage
    int* bad = nullptr;
    std::string err;
};

namespace fvg {
namespace {

// what a face solves (bits 2-3 of its meta word; bits 0-1 the axis; on a boundary face bit 8 set, 4-6 its side and 7 its
// ghost on the right)
constexpr int kFaceR6 = 0;    // WENO5-Z on six entries
constexpr int kFaceR4 = 1;    // four entries (entries 1-4): MUSCL, or WENO3-Z (a WENO5-Z run's faces that hold fewer cells too)
constexpr int kFaceFO = 2;    // first order between two leaves: their conservative states
constexpr int kFaceBnd = 3;   // a boundary face without a reconstruction: the leaf's state and its ghost (round trip with a reconstruction)
constexpr int kCellsNT = 256;

__host__ __device__ inline int ghost_code(int leaf, int side) { return ~(8 * leaf + side); }

struct CellArgs {
    Eos<double> eos;
    Bc bc;
    double shock_blend, weno_eps;
    int limiter;
    long long nleaf, lplane, nface, fplane;
    const double* U;           // [NV][lplane] conservative state the residual is taken of
    const double* W;           // [NV][lplane] its primitive state (runs with a reconstruction)
    const int* code;           // [6][fplane] stencil entries: >= 0 a leaf, < 0 ghost_code(leaf, side)
    const int* meta;           // [fplane]
    double* F;                 // [NV][fplane] face fluxes (per unit measure)
    unsigned long long* smax;  // the bits of the largest face speed
    double *PL, *PR;           // MUSCL-Hancock: [NV][fplane] the face states of the face's left / right side
};

// what the face kernel does with a face's two states: solve the Riemann problem (a residual), keep them for the
// MUSCL-Hancock predictor (CellFluxEngine::fluxes with collect_), or solve it on the predicted states PL / PR
// (CellFluxEngine::predicted_fluxes, CellFluxResidual.cpp:358-392)
constexpr int kFacesFlux = 0, kFacesCollect = 1, kFacesPredicted = 2;

template <int NV> __device__ __forceinline__ St<double, NV> leaf_state(const double* __restrict__ U, long long lplane, long long c) {
    St<double, NV> s;
#pragma unroll
    for (int q = 0; q < NV; ++q) s[q] = U[q * lplane + c];
    return s;
}

template <int NV> __global__ void __launch_bounds__(kCellsNT) k_cells_prim(const Eos<double> e, const double* __restrict__ U, double* __restrict__ W,
                                                                          long long lplane, long long n) {
    const long long c = blockIdx.x * (long long)kCellsNT + threadIdx.x;
    if (c >= n) return;
    const St<double, NV> w = c2p(e, leaf_state<NV>(U, lplane, c));
#pragma unroll
    for (int q = 0; q < NV; ++q) W[q * lplane + c] = w[q];
}

// component q of a stencil entry's primitive state: the leaf's, or the ghost layer cons_to_prim(ghost_state(side, U[leaf]))
template <int NV> __device__ __forceinline__ double entry(const CellArgs& a, int code, int q) {
    if (code >= 0) return a.W[q * a.lplane + code];
    const int g = ~code;
    const St<double, NV> Ug = ghost_state(a.eos, a.bc, g & 7, leaf_state<NV>(a.U, a.lplane, g >> 3));
    return c2p(a.eos, Ug)[q];
}

template <int NV, int RECON, int RIEMANN, int MODE = kFacesFlux>
__global__ void __launch_bounds__(kCellsNT) k_cells_faces(const CellArgs a) {
    __shared__ double red[32];
    const long long f = blockIdx.x * (long long)kCellsNT + threadIdx.x;
    double s = 0.0;
    if (f < a.nface) {
        const int meta = a.meta[f];
        const int axis = meta & 3, kind = (meta >> 2) & 3;
        St<double, NV> UL, UR, F;
        if (MODE == kFacesPredicted) {
            UL = leaf_state<NV>(a.PL, a.fplane, f);
            UR = leaf_state<NV>(a.PR, a.fplane, f);
        } else if (kind == kFaceBnd) {
            const int side = (meta >> 4) & 7;
            const bool ghost_right = (meta >> 7) & 1;
            const St<double, NV> Ui = leaf_state<NV>(a.U, a.lplane, a.code[(ghost_right ? 2 : 3) * a.fplane + f]);
            const St<double, NV> Ug = ghost_state(a.eos, a.bc, side, Ui);
            UL = ghost_right ? Ui : Ug;
            UR = ghost_right ? Ug : Ui;
            if constexpr (RECON != kFirstOrder) {
                UL = round_trip(a.eos, UL);
                UR = round_trip(a.eos, UR);
            }
        } else if (RECON == kFirstOrder || kind == kFaceFO) {
            UL = leaf_state<NV>(a.U, a.lplane, a.code[2 * a.fplane + f]);
            UR = leaf_state<NV>(a.U, a.lplane, a.code[3 * a.fplane + f]);
        } else {
            int cd[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) cd[k] = (kind == kFaceR6 || (k >= 1 && k <= 4)) ? a.code[k * a.fplane + f] : 0;
            St<double, NV> wl, wr;
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                const double c1 = entry<NV>(a, cd[1], q), c2 = entry<NV>(a, cd[2], q), c3 = entry<NV>(a, cd[3], q), c4 = entry<NV>(a, cd[4], q);
                if (RECON == kWeno5 && kind == kFaceR6) {
                    const double c0 = entry<NV>(a, cd[0], q), c5 = entry<NV>(a, cd[5], q);
                    wl[q] = weno5z(c0, c1, c2, c3, c4, a.weno_eps);
                    wr[q] = weno5z(c5, c4, c3, c2, c1, a.weno_eps);
                } else if (RECON == kMuscl) {
                    const double bb = c3 - c2;
                    wl[q] = c2 + 0.5 * limiter(a.limiter, c2 - c1, bb);
                    wr[q] = c3 - 0.5 * limiter(a.limiter, c4 - c3, bb);
                } else {   // WENO3-Z (also the four-entry faces of a WENO5-Z run)
                    wl[q] = weno3z(c1, c2, c3, a.weno_eps);
                    wr[q] = weno3z(c4, c3, c2, a.weno_eps);
                }
            }
            UL = p2c(a.eos, wl);
            UR = p2c(a.eos, wr);
        }
        if constexpr (MODE == kFacesCollect) {
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                a.PL[q * a.fplane + f] = UL[q];
                a.PR[q * a.fplane + f] = UR[q];
            }
        } else {
            const double sf = face_flux<RIEMANN>(a.eos, a.shock_blend, UL, UR, axis, F);
            if (sf > s) s = sf;
#pragma unroll
            for (int q = 0; q < NV; ++q) a.F[q * a.fplane + f] = F[q];
        }
    }
    if constexpr (MODE != kFacesCollect) {
        const double bm = block_max<kCellsNT>(s, red);
        // a non-negative double orders like its bits (a NaN speed never enters: the comparisons above drop it)
        if (threadIdx.x == 0 && bm > 0.0) atomicMax(a.smax, (unsigned long long)__double_as_longlong(bm));
    }
}

// MUSCL-Hancock's predictor of every leaf (CellFluxEngine::predict_cells, CellFluxResidual.cpp:424-470, with
// MusclReconstruction::hancock_cell_2d / 3d, cpp/src/Schemes.cpp:2153-2198): the leaf's limited states on its sides (its
// faces' PR on a low side, PL on a high side) advanced by half_dt times the difference of their own Euler fluxes (the body
// force, with half_dt, joins the difference), each kept where the advanced state is not admissible, and put back on the
// faces; beside a reflecting wall the ghost side of the face is the wall's mirror of the predicted state.
struct PredArgs {
    Eos<double> eos;
    Bc bc;
    long long nleaf, lplane, fplane;
    const double* U;   // the state at the start of the step (the body force of the predictor)
    const int* side_face;
    const int* meta;
    double *PL, *PR;
    double hx, hy, hz, half_dt;
};

template <int DIM, int NV> __global__ void __launch_bounds__(kCellsNT) k_cells_predict(const PredArgs p) {
    const long long c = blockIdx.x * (long long)kCellsNT + threadIdx.x;
    if (c >= p.nleaf) return;
    constexpr int NS = 2 * DIM;
    int fs[NS];
    St<double, NV> st[NS];
#pragma unroll
    for (int sd = 0; sd < NS; ++sd) {
        fs[sd] = p.side_face[NS * c + sd];
        st[sd] = leaf_state<NV>((sd & 1) ? p.PL : p.PR, p.fplane, fs[sd]);   // the high side of a leaf is the left of its face
    }
    St<double, NV> fl[NS];
#pragma unroll
    for (int sd = 0; sd < NS; ++sd) {
        if constexpr (NV == 5)
            fl[sd] = euler_flux3(p.eos, st[sd], sd >> 1);
        else
            fl[sd] = euler_flux2(p.eos, st[sd], sd >> 1);
    }
    St<double, NV> d;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        d[q] = p.hx * (fl[1][q] - fl[0][q]) + p.hy * (fl[3][q] - fl[2][q]);
        if constexpr (DIM == 3) d[q] = d[q] + p.hz * (fl[5][q] - fl[4][q]);
    }
    if (p.bc.grav_on) {
        const St<double, NV> src = body_source<NV>(p.bc, p.U, p.lplane, c);
#pragma unroll
        for (int q = 0; q < NV; ++q) d[q] = d[q] - p.half_dt * src[q];
    }
#pragma unroll
    for (int sd = 0; sd < NS; ++sd) {
        St<double, NV> nst;
#pragma unroll
        for (int q = 0; q < NV; ++q) nst[q] = st[sd][q] - d[q];
        bool ok;
        if constexpr (NV == 5)
            ok = admissible3(p.eos, nst);
        else
            ok = admissible(p.eos, nst);
        if (ok) st[sd] = nst;
        double* mine = (sd & 1) ? p.PL : p.PR;
#pragma unroll
        for (int q = 0; q < NV; ++q) mine[q * p.fplane + fs[sd]] = st[sd][q];
        const int meta = p.meta[fs[sd]];
        if ((meta >> 8) & 1) {
            const int side = (meta >> 4) & 7, type = p.bc.type[side];
            if (type == kBcWall || type == kBcNoSlip || type == kBcMovingWall) {
                const St<double, NV> g = ghost_state(p.eos, p.bc, side, st[sd]);
                double* other = (sd & 1) ? p.PR : p.PL;
#pragma unroll
                for (int q = 0; q < NV; ++q) other[q * p.fplane + fs[sd]] = g[q];
            }
        }
    }
}

// ---- the viscous terms on a 3-D mesh (CellFluxEngine::cell_quantities_3d / viscous_fluxes_3d / viscous_speed_3d,
// CellFluxResidual.cpp:801-972: the expressions of NavierStokes::viscous_residual_3d, so level-0 leaves get its bits)

constexpr int kQ = 13;   // cell quantities per leaf: u, v, w, T, then G[a][b] = du_a/dx_b at 4 + 3 a + b

struct CellVisc {
    ViscArgs va;   // the rules of the diffusive ghost (viscous_ghost_3d): boundary types, u_in, v_in, boundary_order 2
    long long nleaf, lplane, nface, fplane;
    const double* U;
    const int* nbr;     // [6][nleaf] the leaf across each side, -1 at a physical edge
    double* Q;          // [kQ][lplane]
    const int* code;
    const int* meta;
    double* Fv;         // [4][fplane] viscous flux times the face's area: rho u, rho v, rho E, rho w
    double h[3], length[3];
    double mu, k_cond, L, inv_h2;
    int bo2;
    unsigned long long* smax;
};

__global__ void __launch_bounds__(kCellsNT) k_cells_vcells(const CellVisc v) {
    __shared__ double red[32];
    const long long c = blockIdx.x * (long long)kCellsNT + threadIdx.x;
    double s = 0.0;
    if (c < v.nleaf) {
        const St<double, 5> Ui = leaf_state<5>(v.U, v.lplane, c);
        const St<double, 5> W = c2p(v.va.eos, Ui);
        const int mom[3] = {1, 2, 4};
        const double rho = W[0];
        double grad[3][5];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int lo = v.nbr[(2 * b) * v.nleaf + c], hi = v.nbr[(2 * b + 1) * v.nleaf + c];
            const St<double, 5> nl = lo >= 0 ? leaf_state<5>(v.U, v.lplane, lo) : viscous_ghost_3d(v.va, 2 * b, Ui);
            const St<double, 5> nh = hi >= 0 ? leaf_state<5>(v.U, v.lplane, hi) : viscous_ghost_3d(v.va, 2 * b + 1, Ui);
#pragma unroll
            for (int q = 0; q < 5; ++q) grad[b][q] = (nh[q] - nl[q]) / (2.0 * v.h[b]);
        }
        v.Q[3 * v.lplane + c] = W[3] / rho;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double ua = W[mom[a]];
            v.Q[a * v.lplane + c] = ua;
#pragma unroll
            for (int b = 0; b < 3; ++b) v.Q[(4 + 3 * a + b) * v.lplane + c] = (grad[b][mom[a]] - ua * grad[b][0]) / rho;
        }
        // the leaf's viscous speed bound (ViscousBound.hpp: viscous_speed_bound of viscous_nu_eff)
        const double nu_eff = vmax((4.0 / 3.0) * (v.mu / rho), (v.k_cond * (v.va.eos.gamma - 1.0)) / rho) + 1e-12;
        const double vm = vmax(vmax(fabs(W[1]), fabs(W[2])), fabs(W[4]));
        const double sv = vm + sound_speed(v.va.eos, W[3], rho) + 2.0 * v.L * v.inv_h2 * nu_eff;
        if (sv > s) s = sv;
    }
    const double bm = block_max<kCellsNT>(s, red);
    if (threadIdx.x == 0 && bm > 0.0) atomicMax(v.smax, (unsigned long long)__double_as_longlong(bm));
}

// one face normal to axis D (a template parameter, so the pairs below and every array index are constants)
template <int D> __device__ __forceinline__ void cells_vface(const CellVisc& v, long long f, int meta) {
    constexpr int d = D;
    const int mom[3] = {1, 2, 4};
    // the cross derivatives (a, b) = du_a/dx_b a face normal to axis d reads, in the uniform solver's order
    constexpr int pa[4] = {0, 1, 2, D};
    constexpr int pb[4] = {D == 0 ? 1 : 0, D == 1 ? 0 : 1, D == 2 ? 0 : 2, D == 2 ? 1 : 2};
    double vL[3], vR[3], TL, TR, h;
    double Gc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto G = [&](int a, int b, long long c) { return v.Q[(4 + 3 * a + b) * v.lplane + c]; };
    if ((meta >> 8) & 1) {
        const int side = (meta >> 4) & 7;
        const bool ghost_left = !((meta >> 7) & 1);
        const int c = v.code[(ghost_left ? 3 : 2) * v.fplane + f];
        const St<double, 5> Uc = leaf_state<5>(v.U, v.lplane, c);
        const St<double, 5> g = c2p(v.va.eos, viscous_ghost_3d(v.va, side, Uc));
        const double gT = g[3] / g[0];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double gv = g[mom[a]], cv = v.Q[a * v.lplane + c];
            vL[a] = ghost_left ? gv : cv;
            vR[a] = ghost_left ? cv : gv;
        }
        TL = ghost_left ? gT : v.Q[3 * v.lplane + c];
        TR = ghost_left ? v.Q[3 * v.lplane + c] : gT;
        h = v.h[d];
        if (v.bo2) {
            // the tangential difference of the face values (ghost and cell average) of the two neighbours along b; beyond a
            // physical edge along b the neighbour is the leaf's b-ghost and its d-ghost the padded state's edge entry
            double fval[6][3];
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                if (b == d) continue;
#pragma unroll
                for (int hi = 0; hi < 2; ++hi) {
                    const int si = 2 * b + hi;
                    const int code = v.nbr[si * v.nleaf + c];
                    St<double, 5> in, gh;
                    if (code >= 0) {
                        in = leaf_state<5>(v.U, v.lplane, code);
                        gh = viscous_ghost_3d(v.va, side, in);
                    } else {
                        in = viscous_ghost_3d(v.va, si, Uc);
                        gh = d < b ? viscous_ghost_3d(v.va, side, in) : viscous_ghost_3d(v.va, si, viscous_ghost_3d(v.va, side, Uc));
                    }
                    const St<double, 5> Wg = c2p(v.va.eos, gh), Wi = c2p(v.va.eos, in);
#pragma unroll
                    for (int a = 0; a < 3; ++a) fval[si][a] = 0.5 * (Wg[mom[a]] + Wi[mom[a]]);
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) Gc[pa[k]][pb[k]] = (fval[2 * pb[k] + 1][pa[k]] - fval[2 * pb[k]][pa[k]]) / (2.0 * v.h[pb[k]]);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double x = G(pa[k], pb[k], c);
                Gc[pa[k]][pb[k]] = 0.5 * (x + x);
            }
        }
    } else {
        const int L = v.code[2 * v.fplane + f], R = v.code[3 * v.fplane + f];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            vL[a] = v.Q[a * v.lplane + L];
            vR[a] = v.Q[a * v.lplane + R];
        }
        TL = v.Q[3 * v.lplane + L];
        TR = v.Q[3 * v.lplane + R];
        h = 0.5 * (v.h[d] + v.h[d]);
#pragma unroll
        for (int k = 0; k < 4; ++k) Gc[pa[k]][pb[k]] = 0.5 * (G(pa[k], pb[k], L) + G(pa[k], pb[k], R));
    }
    double Gn[3], vf[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        Gn[a] = (vR[a] - vL[a]) / h;
        vf[a] = 0.5 * (vL[a] + vR[a]);
    }
    const double dT = (TR - TL) / h;
    double tau[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a == d) {
            double others = 0.0;
#pragma unroll
            for (int o = 0; o < 3; ++o)
                if (o != d) others += Gc[o][o];
            tau[a] = v.mu * ((4.0 / 3.0) * Gn[d] - (2.0 / 3.0) * others);
        } else {
            tau[a] = v.mu * (Gn[a] + Gc[d][a]);
        }
    }
    const double q_d = -v.k_cond * dT;
    const double area = v.length[d];
    v.Fv[0 * v.fplane + f] = tau[0] * area;
    v.Fv[1 * v.fplane + f] = tau[1] * area;
    v.Fv[2 * v.fplane + f] = (vf[0] * tau[0] + vf[1] * tau[1] + vf[2] * tau[2] - q_d) * area;
    v.Fv[3 * v.fplane + f] = tau[2] * area;
}

__global__ void __launch_bounds__(kCellsNT) k_cells_vfaces(const CellVisc v) {
    const long long f = blockIdx.x * (long long)kCellsNT + threadIdx.x;
    if (f >= v.nface) return;
    const int meta = v.meta[f];
    const int d = meta & 3;
    if (d == 0)
        cells_vface<0>(v, f, meta);
    else if (d == 1)
        cells_vface<1>(v, f, meta);
    else
        cells_vface<2>(v, f, meta);
}

// ---- the viscous terms on a 2-D mesh (CellFluxEngine::cell_quantities / viscous_fluxes / viscous_speed for a quadtree,
// CellFluxResidual.cpp:592-800): u, v, T and the four velocity derivatives per leaf, the x and y face fluxes. The diffusive
// ghost of a 2-D side (BoundaryManager::viscous_ghost) is the 3-D rule with w = 0 (the same momentum rules on rho u and
// rho v, and match_kinetic_energy with a zero w term).
constexpr int kQ2 = 7;   // cell quantities per leaf on a 2-D mesh: u, v, T, du/dx, du/dy, dv/dx, dv/dy

__device__ __forceinline__ St<double, 4> vghost2(const ViscArgs& va, int side, const St<double, 4>& c) {
    St<double, 5> c5;
#pragma unroll
    for (int q = 0; q < 4; ++q) c5[q] = c[q];
    c5[4] = 0.0;
    const St<double, 5> g5 = viscous_ghost_3d(va, side, c5);
    St<double, 4> g;
#pragma unroll
    for (int q = 0; q < 4; ++q) g[q] = g5[q];
    return g;
}

__global__ void __launch_bounds__(kCellsNT) k_cells_vcells2(const CellVisc v) {
    __shared__ double red[32];
    const long long c = blockIdx.x * (long long)kCellsNT + threadIdx.x;
    double s = 0.0;
    if (c < v.nleaf) {
        const St<double, 4> Ui = leaf_state<4>(v.U, v.lplane, c);
        const St<double, 4> W = c2p(v.va.eos, Ui);
        St<double, 4> nb[4];   // left, right, bottom, top (the diffusive ghost at a physical edge)
#pragma unroll
        for (int sd = 0; sd < 4; ++sd) {
            const int code = v.nbr[sd * v.nleaf + c];
            nb[sd] = code >= 0 ? leaf_state<4>(v.U, v.lplane, code) : vghost2(v.va, sd, Ui);
        }
        double gx[3], gy[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            gx[q] = (nb[1][q] - nb[0][q]) / (2.0 * v.h[0]);
            gy[q] = (nb[3][q] - nb[2][q]) / (2.0 * v.h[1]);
        }
        const double rho = W[0], u = W[1], vv = W[2];
        v.Q[0 * v.lplane + c] = u;
        v.Q[1 * v.lplane + c] = vv;
        v.Q[2 * v.lplane + c] = W[3] / rho;
        v.Q[3 * v.lplane + c] = (gx[1] - u * gx[0]) / rho;
        v.Q[4 * v.lplane + c] = (gy[1] - u * gy[0]) / rho;
        v.Q[5 * v.lplane + c] = (gx[2] - vv * gx[0]) / rho;
        v.Q[6 * v.lplane + c] = (gy[2] - vv * gy[0]) / rho;
        const double nu_eff = vmax((4.0 / 3.0) * (v.mu / rho), (v.k_cond * (v.va.eos.gamma - 1.0)) / rho) + 1e-12;
        const double sv = vmax(fabs(W[1]), fabs(W[2])) + sound_speed(v.va.eos, W[3], rho) + 2.0 * v.L * v.inv_h2 * nu_eff;
        if (sv > s) s = sv;
    }
    const double bm = block_max<kCellsNT>(s, red);
    if (threadIdx.x == 0 && bm > 0.0) atomicMax(v.smax, (unsigned long long)__double_as_longlong(bm));
}

__global__ void __launch_bounds__(kCellsNT) k_cells_vfaces2(const CellVisc v) {
    const long long f = blockIdx.x * (long long)kCellsNT + threadIdx.x;
    if (f >= v.nface) return;
    const int meta = v.meta[f];
    const int ax = meta & 3;
    auto Q = [&](int k, long long c) { return v.Q[k * v.lplane + c]; };
    double uL, vL, TL, uR, vR, TR, h, ca, cb;   // ca, cb: the cross derivatives of u and v along the other axis
    if ((meta >> 8) & 1) {
        const int side = (meta >> 4) & 7;
        const bool ghost_left = !((meta >> 7) & 1);
        const int c = v.code[(ghost_left ? 3 : 2) * v.fplane + f];
        const St<double, 4> Uc = leaf_state<4>(v.U, v.lplane, c);
        const St<double, 4> g = c2p(v.va.eos, vghost2(v.va, side, Uc));
        const double gu = g[1], gv = g[2], gT = g[3] / g[0];
        uL = ghost_left ? gu : Q(0, c);
        vL = ghost_left ? gv : Q(1, c);
        TL = ghost_left ? gT : Q(2, c);
        uR = ghost_left ? Q(0, c) : gu;
        vR = ghost_left ? Q(1, c) : gv;
        TR = ghost_left ? Q(2, c) : gT;
        h = v.h[ax];
        if (v.bo2) {
            // the tangential difference of the face values (ghost and cell average) of the two neighbours along the wall; the
            // neighbour across a physical edge of the tangential side is the leaf's ghost on that side, its ghost the corner entry
            const int tl = ax == 0 ? 2 : 0;
            double fu[2], fv[2];
#pragma unroll
            for (int hi = 0; hi < 2; ++hi) {
                const int si = tl + hi;
                const int code = v.nbr[si * v.nleaf + c];
                St<double, 4> in, gh;
                if (code >= 0) {
                    in = leaf_state<4>(v.U, v.lplane, code);
                    gh = vghost2(v.va, side, in);
                } else {
                    in = vghost2(v.va, si, Uc);
                    gh = ax == 0 ? vghost2(v.va, side, in) : vghost2(v.va, si, vghost2(v.va, side, Uc));
                }
                const St<double, 4> Wg = c2p(v.va.eos, gh), Wi = c2p(v.va.eos, in);
                fu[hi] = 0.5 * (Wg[1] + Wi[1]);
                fv[hi] = 0.5 * (Wg[2] + Wi[2]);
            }
            const double h2 = 2.0 * (ax == 0 ? v.h[1] : v.h[0]);
            ca = (fu[1] - fu[0]) / h2;
            cb = (fv[1] - fv[0]) / h2;
        } else {
            const double a = ax == 0 ? Q(4, c) : Q(3, c), b = ax == 0 ? Q(6, c) : Q(5, c);
            ca = 0.5 * (a + a);
            cb = 0.5 * (b + b);
        }
    } else {
        const int L = v.code[2 * v.fplane + f], R = v.code[3 * v.fplane + f];
        uL = Q(0, L);
        vL = Q(1, L);
        TL = Q(2, L);
        uR = Q(0, R);
        vR = Q(1, R);
        TR = Q(2, R);
        h = 0.5 * (v.h[ax] + v.h[ax]);
        ca = ax == 0 ? 0.5 * (Q(4, L) + Q(4, R)) : 0.5 * (Q(3, L) + Q(3, R));
        cb = ax == 0 ? 0.5 * (Q(6, L) + Q(6, R)) : 0.5 * (Q(5, L) + Q(5, R));
    }
    const double u_f = 0.5 * (uL + uR), v_f = 0.5 * (vL + vR);
    const double du_n = (uR - uL) / h, dv_n = (vR - vL) / h, dT_n = (TR - TL) / h;
    const double len = v.length[ax];
    double F1, F2, F3;
    if (ax == 0) {
        const double tau_xx = v.mu * ((4.0 / 3.0) * du_n - (2.0 / 3.0) * cb);
        const double tau_xy = v.mu * (ca + dv_n);
        const double q_x = -v.k_cond * dT_n;
        F1 = tau_xx * len;
        F2 = tau_xy * len;
        F3 = (u_f * tau_xx + v_f * tau_xy - q_x) * len;
    } else {
        const double tau_yy = v.mu * ((4.0 / 3.0) * dv_n - (2.0 / 3.0) * ca);
        const double tau_yx = v.mu * (du_n + cb);
        const double q_y = -v.k_cond * dT_n;
        F1 = tau_yx * len;
        F2 = tau_yy * len;
        F3 = (u_f * tau_yx + v_f * tau_yy - q_y) * len;
    }
    v.Fv[0 * v.fplane + f] = F1;
    v.Fv[1 * v.fplane + f] = F2;
    v.Fv[2 * v.fplane + f] = F3;
}

struct GatherArgs {
    long long nleaf, lplane, fplane;
    const double* F;
    const double* Fv;       // [4][fplane] viscous fluxes times the face area (null: inviscid)
    Bc bc;                  // the body force (bc.grav, when bc.grav_on)
    int hancock;            // MUSCL-Hancock: the predictor's source (the body force from zero) is added as a whole
    const int* side_face;   // [ns * nleaf]: the face on each side of each leaf (one at level 0)
    double length[3], inv_vol;
    int mode;
    double ca, cb;
    double dt;
    const double* U;    // the state the residual was taken of (AXPY, COMBINE)
    const double* U0;   // COMBINE: the state at the start of the step
    double* out;
};

template <int DIM, int NV> __global__ void __launch_bounds__(kCellsNT) k_cells_gather(const GatherArgs g) {
    const long long c = blockIdx.x * (long long)kCellsNT + threadIdx.x;
    if (c >= g.nleaf) return;
    constexpr int NS = 2 * DIM;
    int fs[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) fs[s] = g.side_face[NS * c + s];
    St<double, NV> r;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double G[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) G[s] = g.F[q * g.fplane + fs[s]] * g.length[s >> 1];
        double acc = 0.0 - (G[1] - G[0]);
        acc = acc - (G[3] - G[2]);
        if constexpr (DIM == 3) acc = acc - (G[5] - G[4]);
        r[q] = acc * g.inv_vol;
        if (g.Fv) {   // the viscous terms accumulated: r += (((0 + (H1 - H0)) + (H3 - H2)) + (H5 - H4)) / volume
            double H[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) H[s] = q == 0 ? 0.0 : g.Fv[(q - 1) * g.fplane + fs[s]];
            double vac = 0.0 + (H[1] - H[0]);
            vac = vac + (H[3] - H[2]);
            if constexpr (DIM == 3) vac = vac + (H[5] - H[4]);
            r[q] += vac * g.inv_vol;
        }
    }
    // the body force after the viscous terms (CellFluxEngine::gather, CellFluxResidual.cpp:1015-1024); with MUSCL-Hancock
    // the predictor's source, the body force summed from zero, joins as r + src (:1011-1014)
    if (g.bc.grav_on) {
        if (g.hancock) {
            const St<double, NV> src = body_source<NV>(g.bc, g.U, g.lplane, c);
#pragma unroll
            for (int q = 0; q < NV; ++q) r[q] = r[q] + src[q];
        } else {
            add_body_force<NV>(g.bc, leaf_state<NV>(g.U, g.lplane, c), r);
        }
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        const long long e = q * g.lplane + c;
        double o;
        if (g.mode == kStoreR)
            o = r[q];
        else if (g.mode == kAxpy)
            o = g.U[e] + g.dt * r[q];
        else
            o = g.ca * g.U0[e] + g.cb * (g.U[e] + g.dt * r[q]);
        g.out[e] = o;
    }
}

__global__ void k_cells_in(const double* aos, double* U, long long lplane, long long n, int nvar, int* bad) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        for (int q = 0; q < nvar; ++q) U[q * lplane + c] = aos[5 * c + q];
        if (nvar == 4 && aos[5 * c + 4] != 0.0) atomicOr(bad, 1);
    }
}
__global__ void k_cells_out(const double* U, double* aos, long long lplane, long long n, int nvar) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        for (int q = 0; q < 5; ++q) aos[5 * c + q] = q < nvar ? U[q * lplane + c] : 0.0;
}

// ---- the tables of a level-0 mesh (CellMesh's faces and side lists, CellFluxEngine::build's stencils)

struct Tables {
    long long nface = 0;
    std::vector<int> code[6], meta, side_face;
    std::vector<int> nbr;   // [ns][nleaf]: the leaf across each side (-1 at a physical edge)
};

std::string build_tables(const fvg_config& c, int dim, long long nleaf, const int* ci, const int* cj, const int* ck, Tables& t) {
    const int n3[3] = {c.nx, c.ny, dim == 3 ? c.nz : 1};
    const int ns = 2 * dim;
    std::vector<int> at((size_t)nleaf, -1);
    for (long long l = 0; l < nleaf; ++l) {
        const int p[3] = {ci[l], cj[l], dim == 3 ? ck[l] : 0};
        for (int a = 0; a < 3; ++a)
            if (p[a] < 0 || p[a] >= n3[a]) return "leaf " + std::to_string(l) + " lies outside the base mesh";
        int& slot = at[((size_t)p[2] * n3[1] + p[1]) * n3[0] + p[0]];
        if (slot >= 0) return "leaves " + std::to_string(slot) + " and " + std::to_string(l) + " are the same cell";
        slot = (int)l;
    }
    bool periodic[3];
    for (int a = 0; a < 3; ++a) periodic[a] = c.bc[2 * a] == FVG_BC_PERIODIC;
    // the leaf across side s of leaf l (CellMesh::neighbour): the wrapped cell on a periodic axis, -1 at a physical edge
    auto nbr = [&](int l, int s) -> int {
        int p[3] = {ci[l], cj[l], dim == 3 ? ck[l] : 0};
        const int a = s >> 1;
        p[a] += (s & 1) ? 1 : -1;
        if (p[a] < 0 || p[a] >= n3[a]) {
            if (!periodic[a]) return -1;
            p[a] = (p[a] + n3[a]) % n3[a];
        }
        return at[((size_t)p[2] * n3[1] + p[1]) * n3[0] + p[0]];
    };
    auto beyond = [&](int l, int s) { const int n = nbr(l, s); return n >= 0 ? n : l; };   // edge replication
    const bool muscl = c.reconstruction != FVG_RECON_NONE, weno5 = c.reconstruction == FVG_RECON_WENO5;
    const bool bo2 = muscl && c.boundary_order == 2;
    auto side_ok = [&](int s) { return c.bc[s] != FVG_BC_PERIODIC && c.bc[s] != FVG_BC_NONREFLECTING; };
    t.side_face.assign((size_t)ns * nleaf, -1);
    t.meta.clear();
    for (auto& v : t.code) v.clear();
    auto add = [&](const int e[6], int meta) {
        for (int k = 0; k < 6; ++k) t.code[k].push_back(e[k]);
        t.meta.push_back(meta);
        return (int)t.meta.size() - 1;
    };
    // an interior face between leaves l and r along axis a (CellFluxEngine::face_stencil and far_code for level-0 leaves,
    // with the ghost layers of boundary_order = 2 that CellFluxEngine::fluxes puts in place of replicated leaves)
    auto interior = [&](int l, int r, int a) {
        const int back = 2 * a, fwd = 2 * a + 1;
        int e[6] = {0, 0, l, r, 0, 0};
        if (!muscl) return add(e, a | kFaceFO << 2);
        const int s0 = beyond(l, back), s3 = beyond(r, fwd);
        e[1] = s0;
        e[4] = s3;
        const bool g0 = bo2 && s0 == l && nbr(l, back) == -1 && side_ok(back);
        const bool g3 = bo2 && s3 == r && nbr(r, fwd) == -1 && side_ok(fwd);
        if (g0) e[1] = ghost_code(l, back);
        if (g3) e[4] = ghost_code(r, fwd);
        if (!weno5) return add(e, a | kFaceR4 << 2);
        const int nb0 = nbr(s0, back), nb3 = nbr(s3, fwd);
        const int far0 = s0 == l ? l : (nb0 == -1 ? s0 : nb0);
        const int far1 = s3 == r ? r : (nb3 == -1 ? s3 : nb3);
        e[0] = far0;
        e[5] = far1;
        if (bo2) {
            if (g0)
                e[0] = ghost_code(r, back);
            else if (far0 == s0 && nb0 == -1 && side_ok(back))
                e[0] = ghost_code(s0, back);
            if (g3)
                e[5] = ghost_code(l, fwd);
            else if (far1 == s3 && nb3 == -1 && side_ok(fwd))
                e[5] = ghost_code(s3, fwd);
        }
        return add(e, a | kFaceR6 << 2);
    };
    // a face on physical side sd of leaf l (the boundary branch of CellFluxEngine::fluxes)
    auto boundary = [&](int l, int sd) {
        const int a = sd >> 1;
        const bool gr = (sd & 1) != 0;   // the ghost on the right: the mesh's high side
        const int bside = sd << 4 | (gr ? 1 : 0) << 7 | 1 << 8;   // every boundary face carries its side (the viscous pass reads it)
        const int bmeta = a | kFaceBnd << 2 | bside;
        int e[6] = {0, 0, gr ? l : 0, gr ? 0 : l, 0, 0};
        if (!bo2 || !side_ok(sd)) return add(e, bmeta);
        const int n1 = nbr(l, sd ^ 1);
        if (n1 < 0) return add(e, bmeta);
        int n2 = weno5 ? nbr(n1, sd ^ 1) : -1;
        if (n2 < 0) n2 = -1;
        if (n2 >= 0) {
            const int hi[6] = {n2, n1, l, ghost_code(l, sd), ghost_code(n1, sd), ghost_code(n2, sd)};
            const int lo[6] = {ghost_code(n2, sd), ghost_code(n1, sd), ghost_code(l, sd), l, n1, n2};
            return add(gr ? hi : lo, a | kFaceR6 << 2 | bside);
        }
        const int hi[6] = {0, n1, l, ghost_code(l, sd), ghost_code(n1, sd), 0};
        const int lo[6] = {0, ghost_code(n1, sd), ghost_code(l, sd), l, n1, 0};
        return add(gr ? hi : lo, a | kFaceR4 << 2 | bside);
    };
    // faces in leaf order (a leaf makes the face on its low side of every axis, and the one on its high side at a
    // physical edge), so the faces of neighbouring leaves sit close together too
    for (long long l = 0; l < nleaf; ++l) {
        for (int a = 0; a < dim; ++a) {
            const int lo = nbr((int)l, 2 * a);
            const int f = lo >= 0 ? interior(lo, (int)l, a) : boundary((int)l, 2 * a);
            t.side_face[(size_t)ns * l + 2 * a] = f;
            if (lo >= 0) t.side_face[(size_t)ns * lo + 2 * a + 1] = f;
            if (nbr((int)l, 2 * a + 1) < 0) t.side_face[(size_t)ns * l + 2 * a + 1] = boundary((int)l, 2 * a + 1);
        }
    }
    t.nface = (long long)t.meta.size();
    t.nbr.resize((size_t)ns * nleaf);
    for (int sd = 0; sd < ns; ++sd)
        for (long long l = 0; l < nleaf; ++l) t.nbr[(size_t)sd * nleaf + l] = nbr((int)l, sd);
    for (int v : t.side_face)
        if (v < 0) return "a leaf side without a face (the leaves do not tile the base mesh)";
    return "";
}

int fail(fvg_cells* e, int code, const std::string& msg) {
    e->err = msg;
    return code;
}

#define CKC(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(e, FVG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int flat_blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

template <int NV, int MODE = kFacesFlux> cudaError_t launch_faces(const fvg_cells* e, const CellArgs& a) {
    const int blocks = (int)((a.nface + kCellsNT - 1) / kCellsNT);
    const int recon = e->cfg.reconstruction, lm = e->cfg.riemann == FVG_RIEMANN_LOWMACH;
#define FACES(R)                                                                                            \
    if (lm)                                                                                                 \
        k_cells_faces<NV, R, kLowMach, MODE><<<blocks, kCellsNT, 0, e->stream>>>(a);                        \
    else                                                                                                    \
        k_cells_faces<NV, R, kHLLC, MODE><<<blocks, kCellsNT, 0, e->stream>>>(a);
    switch (recon) {
    case FVG_RECON_NONE: FACES(kFirstOrder) break;
    case FVG_RECON_MUSCL: FACES(kMuscl) break;
    case FVG_RECON_WENO3: FACES(kWeno3) break;
    default: FACES(kWeno5) break;
    }
#undef FACES
    return cudaGetLastError();
}

// one residual of Uin (its largest face speed into smax[slot]), gathered into out with the stage update `mode`; with
// half_dt > 0 the residual of MUSCL-Hancock (the face states predicted by half_dt first, CellAdvance::advance with
// CellFluxEngine::predict_level and compute_level_fluxes(predicted), cpp/src/CellAdvance.cpp)
int residual_pass(fvg_cells* e, const double* Uin, int slot, int mode, double ca, double cb, double dt, const double* U0, double* out,
                  double half_dt = 0.0) {
    const long long n = e->nleaf;
    CKC(cudaMemsetAsync(e->smax + slot, 0, sizeof(unsigned long long), e->stream));
    if (e->cfg.reconstruction != FVG_RECON_NONE) {
        const int blocks = (int)((n + kCellsNT - 1) / kCellsNT);
        if (e->nvar == 5)
            k_cells_prim<5><<<blocks, kCellsNT, 0, e->stream>>>(e->eos, Uin, e->W, e->lplane, n);
        else
            k_cells_prim<4><<<blocks, kCellsNT, 0, e->stream>>>(e->eos, Uin, e->W, e->lplane, n);
        CKC(cudaGetLastError());
    }
    CellArgs a{};
    a.eos = e->eos;
    a.bc = e->bc;
    a.shock_blend = e->cfg.shock_blend;
    a.weno_eps = e->cfg.weno_epsilon;
    a.limiter = e->cfg.limiter;
    a.nleaf = n;
    a.lplane = e->lplane;
    a.nface = e->nface;
    a.fplane = e->fplane;
    a.U = Uin;
    a.W = e->W;
    a.code = e->code;
    a.meta = e->meta;
    a.F = e->F;
    a.smax = e->smax + slot;
    a.PL = e->PL;
    a.PR = e->PR;
    if (half_dt > 0.0) {   // the limited face states, the prediction of every leaf, the Riemann problems on the predicted states
        CKC((e->nvar == 5 ? launch_faces<5, kFacesCollect>(e, a) : launch_faces<4, kFacesCollect>(e, a)));
        PredArgs pa{};
        pa.eos = e->eos;
        pa.bc = e->bc;
        pa.nleaf = n;
        pa.lplane = e->lplane;
        pa.fplane = e->fplane;
        pa.U = Uin;
        pa.side_face = e->side_face;
        pa.meta = e->meta;
        pa.PL = e->PL;
        pa.PR = e->PR;
        pa.hx = half_dt / e->h[0];   // hx = half_dt / dx, as the uniform solver's predictor
        pa.hy = half_dt / e->h[1];
        pa.hz = e->dim == 3 ? half_dt / e->h[2] : 0.0;
        pa.half_dt = half_dt;
        const int bl = (int)((n + kCellsNT - 1) / kCellsNT);
        if (e->dim == 3)
            k_cells_predict<3, 5><<<bl, kCellsNT, 0, e->stream>>>(pa);
        else
            k_cells_predict<2, 4><<<bl, kCellsNT, 0, e->stream>>>(pa);
        CKC(cudaGetLastError());
        CKC((e->nvar == 5 ? launch_faces<5, kFacesPredicted>(e, a) : launch_faces<4, kFacesPredicted>(e, a)));
    } else {
        CKC(e->nvar == 5 ? launch_faces<5>(e, a) : launch_faces<4>(e, a));
    }
    if (e->visc) {   // the cell quantities and the leaves' speed bounds, then the viscous face fluxes
        CellVisc v{};
        v.va.eos = e->eos;
        v.va.bc = e->bc;
        v.va.u_in = e->cfg.u_in;
        v.va.v_in = e->cfg.v_in;
        v.va.bface2 = e->cfg.boundary_order == 2;
        v.nleaf = n;
        v.lplane = e->lplane;
        v.nface = e->nface;
        v.fplane = e->fplane;
        v.U = Uin;
        v.nbr = e->nbr;
        v.Q = e->Q;
        v.code = e->code;
        v.meta = e->meta;
        v.Fv = e->Fv;
        for (int k = 0; k < 3; ++k) {
            v.h[k] = e->h[k];
            v.length[k] = e->length[k];
        }
        v.mu = e->mu;
        v.k_cond = e->k_cond;
        v.L = e->L;
        v.inv_h2 = e->inv_h2;
        v.bo2 = e->cfg.boundary_order == 2;
        v.smax = e->smax + slot;
        const int bl = (int)((n + kCellsNT - 1) / kCellsNT), bf = (int)((e->nface + kCellsNT - 1) / kCellsNT);
        if (e->dim == 3) {
            k_cells_vcells<<<bl, kCellsNT, 0, e->stream>>>(v);
            CKC(cudaGetLastError());
            k_cells_vfaces<<<bf, kCellsNT, 0, e->stream>>>(v);
        } else {
            k_cells_vcells2<<<bl, kCellsNT, 0, e->stream>>>(v);
            CKC(cudaGetLastError());
            k_cells_vfaces2<<<bf, kCellsNT, 0, e->stream>>>(v);
        }
        CKC(cudaGetLastError());
    }
    GatherArgs g{};
    g.nleaf = n;
    g.lplane = e->lplane;
    g.fplane = e->fplane;
    g.F = e->F;
    g.Fv = e->visc ? e->Fv : nullptr;
    g.bc = e->bc;
    g.hancock = half_dt > 0.0;
    g.side_face = e->side_face;
    for (int k = 0; k < 3; ++k) g.length[k] = e->length[k];
    g.inv_vol = e->inv_vol;
    g.mode = mode;
    g.ca = ca;
    g.cb = cb;
    g.dt = dt;
    g.U = Uin;
    g.U0 = U0;
    g.out = out;
    const int blocks = (int)((n + kCellsNT - 1) / kCellsNT);
    if (e->dim == 3)
        k_cells_gather<3, 5><<<blocks, kCellsNT, 0, e->stream>>>(g);
    else
        k_cells_gather<2, 4><<<blocks, kCellsNT, 0, e->stream>>>(g);
    CKC(cudaGetLastError());
    return FVG_OK;
}

int read_speed(fvg_cells* e, int slot, double* smax) {
    unsigned long long bits = 0;
    CKC(cudaMemcpyAsync(&bits, e->smax + slot, sizeof bits, cudaMemcpyDeviceToHost, e->stream));
    CKC(cudaStreamSynchronize(e->stream));
    double v;
    std::memcpy(&v, &bits, sizeof v);
    if (smax) *smax = v;
    return FVG_OK;
}

}   // namespace
}   // namespace fvg

using namespace fvg;

extern "C" {

int fvg_cells_create(const fvg_config* cfg, int nleaf, const int* level, const int* ci, const int* cj, const int* ck, fvg_cells** out) {
    std::string* cerr = create_error_slot();
    if (!cfg || !out || !level || !ci || !cj || (cfg->nz > 1 && !ck)) {
        *cerr = "null argument";
        return FVG_ERR_ARGUMENT;
    }
    *out = nullptr;
    const fvg_config& c = *cfg;
    std::string why = config_error(c);
    const char* no = nullptr;
    if (c.use_ibm) no = "an immersed body";
    else if (config_has_expressions(c)) no = "source terms and time-dependent boundary values";
    else if (c.positivity_fallback) no = "positivity_fallback";
    else if (c.flux_quadrature == 1) no = "flux_quadrature = fourth";
    else if (c.precision != FVG_PREC_FP64) no = "the mixed-precision form";
    for (int s = 0; s < 6 && !no; ++s)
        if (c.bc[s] == FVG_BC_NONREFLECTING || c.bc[s] == FVG_BC_MASSFLOWINLET) no = "non-reflecting outlets and mass-flow inlets";
    if (why.empty() && no) why = std::string("the cell engine on the device does not take ") + no + " yet";
    const long long ncell = (long long)c.nx * c.ny * c.nz;
    if (why.empty() && (long long)nleaf != ncell) why = "the leaves do not tile the base mesh (" + std::to_string(nleaf) + " leaves, " + std::to_string(ncell) + " cells)";
    if (why.empty() && ncell >= (1LL << 28)) why = "more than 2^28 leaves";
    for (int l = 0; why.empty() && l < nleaf; ++l)
        if (level[l] != 0) why = "leaf " + std::to_string(l) + " is of level " + std::to_string(level[l]) + ": only level-0 leaves are built on the device";
    if (!why.empty()) {
        *cerr = why;
        return FVG_ERR_CONFIG;
    }
    auto* e = new fvg_cells();
    e->cfg = c;
    e->dim = c.nz > 1 ? 3 : 2;
    e->nvar = e->dim == 3 ? 5 : 4;
    e->ns = 2 * e->dim;
    e->nleaf = nleaf;
    e->lplane = (e->nleaf + 31) / 32 * 32;
    Tables t;
    why = build_tables(c, e->dim, nleaf, ci, cj, ck, t);
    if (!why.empty()) {
        delete e;
        *cerr = why;
        return FVG_ERR_CONFIG;
    }
    e->nface = t.nface;
    e->fplane = (t.nface + 31) / 32 * 32;
    e->eos.type = c.eos_type;
    e->eos.gamma = c.gamma;
    e->eos.p_inf = c.p_inf;
    for (int s = 0; s < 6; ++s) e->bc.type[s] = c.bc[s];
    e->bc.u_in = c.u_in;
    e->bc.v_in = c.v_in;
    e->bc.p_out = c.p_out;
    const double dx = c.Lx / c.nx, dy = c.Ly / c.ny, dz = c.Lz / c.nz;   // CellMesh::dx(0) ... (CellMesh.cpp:39-67)
    e->visc = c.use_viscous != 0;
    e->h[0] = dx;
    e->h[1] = dy;
    e->h[2] = dz;
    e->mu = c.mu;
    e->k_cond = c.mu * c.gamma / (c.pr * (c.gamma - 1.0));                          // TransportLaw (Core.hpp:194-197)
    if (e->dim == 3) {
        e->L = 2.0 / (1.0 / dx + 1.0 / dy + 1.0 / dz);                              // step_length_3d
        e->inv_h2 = 1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz);            // inv_h2_3d
    } else {
        e->L = vmin(dx, dy);                                                         // step_length_2d
        e->inv_h2 = 1.0 / (dx * dx) + 1.0 / (dy * dy);                              // inv_h2_2d
    }
    e->bc.grav_on = c.use_bodyforce ? 1 : 0;   // ConstantBodyForce (gz only on a 3-D mesh)
    e->bc.grav[0] = c.use_bodyforce ? c.gx : 0.0;
    e->bc.grav[1] = c.use_bodyforce ? c.gy : 0.0;
    e->bc.grav[2] = c.use_bodyforce && e->dim == 3 ? c.gz : 0.0;
    if (e->dim == 3) {
        e->length[0] = dy * dz;
        e->length[1] = dx * dz;
        e->length[2] = dx * dy;
        e->inv_vol = 1.0 / (dx * dy * dz);
    } else {
        e->length[0] = dy;
        e->length[1] = dx;
        e->inv_vol = 1.0 / (dx * dy);
    }
    auto bail = [&](const char* what, cudaError_t err) {
        *cerr = std::string(what) + ": " + cudaGetErrorString(err);
        fvg_cells_destroy(e);
        return FVG_ERR_CUDA;
    };
    cudaError_t err = cudaSetDevice(c.device);
    if (err != cudaSuccess) return bail("cudaSetDevice", err);
    if ((err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail("stream", err);
    const size_t lb = sizeof(double) * e->nvar * e->lplane, fb = sizeof(double) * e->nvar * e->fplane;
    const bool rec = c.reconstruction != FVG_RECON_NONE;
    if ((err = cudaMalloc(&e->U, lb)) != cudaSuccess || (err = cudaMalloc(&e->Ut, lb)) != cudaSuccess || (err = cudaMalloc(&e->R, lb)) != cudaSuccess ||
        (rec && (err = cudaMalloc(&e->W, lb)) != cudaSuccess) || (err = cudaMalloc(&e->F, fb)) != cudaSuccess ||
        (err = cudaMalloc(&e->code, sizeof(int) * 6 * e->fplane)) != cudaSuccess || (err = cudaMalloc(&e->meta, sizeof(int) * e->fplane)) != cudaSuccess ||
        (err = cudaMalloc(&e->side_face, sizeof(int) * e->ns * e->nleaf)) != cudaSuccess ||
        (err = cudaMalloc(&e->smax, sizeof(unsigned long long) * 3)) != cudaSuccess || (err = cudaMalloc(&e->bad, sizeof(int))) != cudaSuccess)
        return bail("cudaMalloc", err);
    if (c.time_scheme == FVG_TS_HANCOCK &&
        ((err = cudaMalloc(&e->PL, fb)) != cudaSuccess || (err = cudaMalloc(&e->PR, fb)) != cudaSuccess))
        return bail("cudaMalloc", err);
    if (e->visc) {
        if ((err = cudaMalloc(&e->nbr, sizeof(int) * t.nbr.size())) != cudaSuccess || (err = cudaMalloc(&e->Q, sizeof(double) * (e->dim == 3 ? kQ : kQ2) * e->lplane)) != cudaSuccess ||
            (err = cudaMalloc(&e->Fv, sizeof(double) * 4 * e->fplane)) != cudaSuccess)
            return bail("cudaMalloc", err);
        if ((err = cudaMemcpy(e->nbr, t.nbr.data(), sizeof(int) * t.nbr.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return bail("cudaMemcpy", err);
    }
    for (int k = 0; k < 6; ++k)
        if ((err = cudaMemcpy(e->code + k * e->fplane, t.code[k].data(), sizeof(int) * e->nface, cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail("cudaMemcpy", err);
    if ((err = cudaMemcpy(e->meta, t.meta.data(), sizeof(int) * e->nface, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (err = cudaMemcpy(e->side_face, t.side_face.data(), sizeof(int) * t.side_face.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (err = cudaMemset(e->U, 0, lb)) != cudaSuccess || (err = cudaMemset(e->Ut, 0, lb)) != cudaSuccess)
        return bail("cudaMemcpy", err);
    *out = e;
    return FVG_OK;
}

int fvg_cells_destroy(fvg_cells* e) {
    if (!e) return FVG_OK;
    cudaSetDevice(e->cfg.device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (void* p : {(void*)e->U, (void*)e->Ut, (void*)e->W, (void*)e->R, (void*)e->F, (void*)e->staging, (void*)e->code, (void*)e->meta,
                    (void*)e->side_face, (void*)e->smax, (void*)e->bad, (void*)e->nbr, (void*)e->Q, (void*)e->Fv, (void*)e->PL, (void*)e->PR})
        if (p) cudaFree(p);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return FVG_OK;
}

const char* fvg_cells_last_error(const fvg_cells* e) { return e ? e->err.c_str() : "null handle"; }

int fvg_cells_info(const fvg_cells* e, long long* nleaf, long long* nface) {
    if (!e) return FVG_ERR_ARGUMENT;
    if (nleaf) *nleaf = e->nleaf;
    if (nface) *nface = e->nface;
    return FVG_OK;
}

static int cells_staging(fvg_cells* e) {
    if (!e->staging) CKC(cudaMalloc(&e->staging, sizeof(double) * 5 * e->nleaf));
    return FVG_OK;
}

int fvg_cells_upload_state(fvg_cells* e, const double* U, size_t nleaf) {
    if (!e || !U) return FVG_ERR_ARGUMENT;
    if ((long long)nleaf != e->nleaf) return fail(e, FVG_ERR_ARGUMENT, "nleaf is not the mesh's");
    CKC(cudaSetDevice(e->cfg.device));
    int rc = cells_staging(e);
    if (rc) return rc;
    CKC(cudaMemcpyAsync(e->staging, U, sizeof(double) * 5 * nleaf, cudaMemcpyHostToDevice, e->stream));
    CKC(cudaMemsetAsync(e->bad, 0, sizeof(int), e->stream));
    k_cells_in<<<flat_blocks(e->nleaf), 256, 0, e->stream>>>(e->staging, e->U, e->lplane, e->nleaf, e->nvar, e->bad);
    CKC(cudaGetLastError());
    int hbad = 0;
    CKC(cudaMemcpyAsync(&hbad, e->bad, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    CKC(cudaStreamSynchronize(e->stream));
    if (hbad) return fail(e, FVG_ERR_STATE, "rho w must be zero on a 2-D mesh");
    return FVG_OK;
}

static int cells_download(fvg_cells* e, const double* planes, double* U, size_t nleaf) {
    if (!e || !U) return FVG_ERR_ARGUMENT;
    if ((long long)nleaf != e->nleaf) return fail(e, FVG_ERR_ARGUMENT, "nleaf is not the mesh's");
    CKC(cudaSetDevice(e->cfg.device));
    int rc = cells_staging(e);
    if (rc) return rc;
    k_cells_out<<<flat_blocks(e->nleaf), 256, 0, e->stream>>>(planes, e->staging, e->lplane, e->nleaf, e->nvar);
    CKC(cudaGetLastError());
    CKC(cudaMemcpyAsync(U, e->staging, sizeof(double) * 5 * nleaf, cudaMemcpyDeviceToHost, e->stream));
    CKC(cudaStreamSynchronize(e->stream));
    return FVG_OK;
}

int fvg_cells_download_state(fvg_cells* e, double* U, size_t nleaf) { return e ? cells_download(e, e->U, U, nleaf) : FVG_ERR_ARGUMENT; }

int fvg_cells_residual(fvg_cells* e, double* R, size_t nleaf, double* smax) {
    if (!e || !R) return FVG_ERR_ARGUMENT;
    if ((long long)nleaf != e->nleaf) return fail(e, FVG_ERR_ARGUMENT, "nleaf is not the mesh's");
    CKC(cudaSetDevice(e->cfg.device));
    int rc = residual_pass(e, e->U, 0, kStoreR, 0.0, 0.0, 0.0, nullptr, e->R);
    if (!rc) rc = read_speed(e, 0, smax);
    if (!rc) rc = cells_download(e, e->R, R, nleaf);
    return rc;
}

// The stages of one step of fixed length dt (TimeScheme::advance_fixed_dt, cpp/src/TimeScheme.cpp:100-290), enqueued on
// the engine's stream; the first stage's largest face speed lands in smax[0].
static int cells_enqueue_step(fvg_cells* e, double dt) {
    const int ts = e->cfg.time_scheme;
    int rc;
    if (ts == FVG_TS_EULER) return residual_pass(e, e->U, 0, kAxpy, 0.0, 0.0, dt, nullptr, e->U);
    if (ts == FVG_TS_HANCOCK) return residual_pass(e, e->U, 0, kAxpy, 0.0, 0.0, dt, nullptr, e->U, 0.5 * dt);
    if ((rc = residual_pass(e, e->U, 0, kAxpy, 0.0, 0.0, dt, nullptr, e->Ut))) return rc;   // U1 = U + dt R(U)
    if (ts == FVG_TS_SSPRK2) return residual_pass(e, e->Ut, 1, kCombine, 0.5, 0.5, dt, e->U, e->U);
    if ((rc = residual_pass(e, e->Ut, 1, kCombine, 0.75, 0.25, dt, e->U, e->Ut))) return rc;
    return residual_pass(e, e->Ut, 2, kCombine, 1.0 / 3.0, 2.0 / 3.0, dt, e->U, e->U);
}

int fvg_cells_step(fvg_cells* e, double dt, double t, double* smax) {
    (void)t;   // the stage times matter to time-dependent terms only, which the engine does not take
    if (!e) return FVG_ERR_ARGUMENT;
    CKC(cudaSetDevice(e->cfg.device));
    int rc = cells_enqueue_step(e, dt);
    if (!rc) rc = read_speed(e, 0, smax);
    return rc;
}

int fvg_cells_advance(fvg_cells* e, double dt, int nsteps, double* smax) {
    if (!e || nsteps < 0) return FVG_ERR_ARGUMENT;
    CKC(cudaSetDevice(e->cfg.device));
    for (int k = 0; k < nsteps; ++k) {
        const int rc = cells_enqueue_step(e, dt);
        if (rc) return rc;
    }
    return read_speed(e, 0, smax);
}

int fvg_cells_stream(fvg_cells* e, void** stream) {
    if (!e || !stream) return FVG_ERR_ARGUMENT;
    *stream = e->stream;
    return FVG_OK;
}

}   // extern "C"
