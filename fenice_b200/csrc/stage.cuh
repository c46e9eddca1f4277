// The fused stage kernel: reconstruction (MUSCL / WENO3-Z / WENO5-Z or first order) + Riemann solver + flux
// balance + the time-integrator update of one Runge-Kutta stage, on a tile of cells per CTA.
//
// The reference makes one pass per row (2-D) or plane (3-D) over the mesh (fused_residual_2d / 3d,
// cpp/src/Schemes.cpp:1069-1183); here a CTA owns a TX x TY x TZ tile and sweeps its axes in turn. Per axis:
//   1. load:   the primitive state of the tile extended by H cells along the axis (H = 3 for WENO5-Z, else 2)
//              into shared memory, boundary conditions applied by index mapping (stencil_cons), one
//              cons_to_prim per cell;
//   2. recon:  one thread per (face, variable) computes the left and right face values;
//   3. flux:   one thread per face converts them to conservative form and solves the Riemann problem (faces of a
//              side without a halo take the first-order side states through the round trip instead);
//   4. balance: one thread per cell adds the face-flux difference of this axis to a shared-memory accumulator,
//              in the reference's expression order ((0 - x) - y) - z, so the result has its bits.
// The faces between two tiles are solved by both (the same bits; the reference's thread blocks do the same).
// Epilogue: R = acc * (1 / volume) (+ the viscous residual of the stage, + the body force), then the stage update
//   STORE_R:  out = R
//   AXPY:     out = U + dt R                            (forward Euler, MUSCL-Hancock)
//   COMBINE:  out = a U0 + b (U + dt R)                 (SSP-RK2 / RK3 stages 2 and 3)
// with dt read from the device control block. Each CTA writes the largest face wave speed it saw.
#pragma once

#include "grid.cuh"

namespace fvg {

constexpr int kStoreR = 0, kAxpy = 1, kCombine = 2;

struct StageArgs {
    Mesh m;
    Bc bc;
    Eos<double> eos;
    double shock_blend, weno_eps;
    int limiter;
    int mode;
    double ca, cb;              // COMBINE coefficients
    const double* U;            // the state the residual is taken of (read with halos)
    const double* U0;           // COMBINE: the state at the start of the step (read at the cell only)
    double* out;                // R or the updated state (never aliases U; may alias U0)
    const double* Rv;           // viscous residual to add (null: none)
    // the 3-D mixed form's viscous balance sums instead (FP32, the planes rho u .. rho w after the density's, whose
    // viscous term is 0): the viscous residual is each sum widened to FP64 times 1 / volume (null: none)
    const float* Rvf;
    double* blockmax;           // per-CTA largest wave speed
    const Ctl* ctl;             // dt
    const int* gate;            // the kernel does nothing unless *gate (the control block's `active` or `seed`)
    int tiles[3];               // tiles per axis
    int b0;                     // the tile of the launch's first CTA (a launch over a range of tiles; 0: all)
    // the learned troubled-cell sensor's tile flags (mixed-precision WENO5-Z kernels with the sensor only): one byte per
    // axis and tile (axis-major), 1 where the tile's reconstructions along the axis stay WENO5-Z, 0 where they are linear
    const unsigned char* sens_flags;
    // positivity_fallback: the cells flagged in this stage (null: none); a face next to one takes the cells' states
    const unsigned char* fb;
    // the TMA tensor maps of U for the three sweeps (a host address of TmaMaps, tma.cuh; null: the index-mapping loader
    // only): the launch of a kernel that stages interior tiles by TMA passes them as a kernel parameter
    const void* tma;
};

// positivity_fallback's flag of a stencil position (Schemes.cpp:548-557): the cell's; across a periodic seam the wrapped
// cell's; beyond any other side none (a ghost layer is never flagged).
template <int DIM> __device__ __forceinline__ bool fb_flagged(const Mesh& m, const Bc& bc, const unsigned char* fb, int i, int j, int k) {
    int p[3] = {i, j, k};
    const int n3[3] = {m.nx, m.ny, m.nz};
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        if (p[a] >= 0 && p[a] < n3[a]) continue;
        if (bc.halo[2 * a + (p[a] < 0 ? 0 : 1)] != kHaloWrap) return false;
        p[a] = p[a] < 0 ? p[a] + n3[a] : p[a] - n3[a];
    }
    return fb[((long long)p[2] * m.ny + p[1]) * m.nx + p[0]] != 0;
}

template <int DIM, int RECON, int TX, int TY, int TZ> struct StageShape {
    static constexpr int NV = DIM == 3 ? 5 : 4;
    static constexpr int H = RECON == kWeno5 ? 3 : (RECON == kFirstOrder ? 1 : 2);
    static constexpr int NC = TX * TY * TZ;
    static constexpr int T3[3] = {TX, TY, TZ};
    static constexpr int ext(int a) { return (T3[0] + (a == 0 ? 2 * H : 0)) * (T3[1] + (a == 1 ? 2 * H : 0)) * (T3[2] + (a == 2 ? 2 * H : 0)); }
    static constexpr int nf(int a) { return (T3[0] + (a == 0)) * (T3[1] + (a == 1)) * (T3[2] + (a == 2)); }
    static constexpr int cmax(int a, int b) { return a > b ? a : b; }
    static constexpr int EXT = cmax(cmax(ext(0), ext(1)), DIM == 3 ? ext(2) : 0);
    static constexpr int NF = cmax(cmax(nf(0), nf(1)), DIM == 3 ? nf(2) : 0);
    // shared memory (doubles): P [NV][EXT] primitive stencil, WL / WR [NV][NF] face values (the fluxes overwrite WL),
    // acc [NV][NC] the balance, 32 for the reduction
    static constexpr int P_SIZE = NV * EXT;
    static constexpr int SMEM_DOUBLES = P_SIZE + 2 * NV * NF + NV * NC + 32;
    static constexpr int FLAG_BYTES = (EXT + 7) / 8 * 8;   // solidity of the extended tile (WENO5-Z beside an immersed body)
    static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES + FLAG_BYTES;
};

// One axis of the tile sweep of stage_kernel (the axis a template parameter, so the extents of the extended tile and of
// the face grid are compile-time constants).
template <int AXIS, int DIM, int RECON, int RIEMANN, int TX, int TY, int TZ, int NT, bool FULL = true>
__device__ __forceinline__ void stage_axis(const StageArgs& a, double* __restrict__ P, double* __restrict__ WL, double* __restrict__ WR,
                                           double* __restrict__ acc, unsigned char* __restrict__ Sf, const int o3[3], double& smax) {
    using S = StageShape<DIM, RECON, TX, TY, TZ>;
    constexpr int NV = S::NV, H = S::H, NC = S::NC;
    constexpr int axis = AXIS;
    const Mesh& m = a.m;
    const int tid = threadIdx.x;
    const int n3[3] = {m.nx, m.ny, m.nz};
    {
        // extents of the extended tile and of the face grid of this axis (x fastest)
        constexpr int E[3] = {TX + (AXIS == 0 ? 2 * H : 0), TY + (AXIS == 1 ? 2 * H : 0), TZ + (AXIS == 2 ? 2 * H : 0)};
        constexpr int Fd[3] = {TX + (AXIS == 0), TY + (AXIS == 1), TZ + (AXIS == 2)};
        constexpr int nE = E[0] * E[1] * E[2], nF = Fd[0] * Fd[1] * Fd[2];
        // ---- 1. load (primitive; first order keeps the conservative state)
        for (int e = tid; e < nE; e += NT) {
            int l3[3] = {e % E[0], (e / E[0]) % E[1], e / (E[0] * E[1])};
            l3[axis] -= H;
            const St<double, NV> u = stencil_cons<DIM, NV, FULL>(m, a.bc, a.eos, a.U, o3[0] + l3[0], o3[1] + l3[1], o3[2] + l3[2]);
            if constexpr (RECON == kWeno5)
                if (a.bc.solid) Sf[e] = stencil_solid<DIM>(m, a.bc, o3[0] + l3[0], o3[1] + l3[1], o3[2] + l3[2]);
            if constexpr (RECON == kFirstOrder) {
#pragma unroll
                for (int q = 0; q < NV; ++q) P[q * S::EXT + e] = u[q];
            } else {
                const St<double, NV> w = c2p(a.eos, u);
#pragma unroll
                for (int q = 0; q < NV; ++q) P[q * S::EXT + e] = w[q];
            }
        }
        __syncthreads();
        // stride of the stencil along the axis in the extended tile, and the extended position of face f's first cell
        const int sstride = axis == 0 ? 1 : (axis == 1 ? E[0] : E[0] * E[1]);
        // ---- 2. face values
        if constexpr (RECON != kFirstOrder) {
            for (int it = tid; it < nF * NV; it += NT) {
                const int f = it % nF, q = it / nF;
                const int f3[3] = {f % Fd[0], (f / Fd[0]) % Fd[1], f / (Fd[0] * Fd[1])};
                // face t (local, between cells t-1 and t) has its stencil at extended positions t .. t + 2H - 1
                const int base = (f3[2] * E[1] + f3[1]) * E[0] + f3[0];
                const double* c = P + q * S::EXT + base;
                double wl, wr;
                if constexpr (RECON == kMuscl) {
                    const double c0 = c[0], c1 = c[sstride], c2 = c[2 * sstride], c3 = c[3 * sstride];
                    const double bb = c2 - c1;
                    wl = c1 + 0.5 * limiter(a.limiter, c1 - c0, bb);
                    wr = c2 - 0.5 * limiter(a.limiter, c3 - c2, bb);
                } else if constexpr (RECON == kWeno3) {
                    wl = weno3z(c[0], c[sstride], c[2 * sstride], a.weno_eps);
                    wr = weno3z(c[3 * sstride], c[2 * sstride], c[sstride], a.weno_eps);
                } else {
                    const double c0 = c[0], c1 = c[sstride], c2 = c[2 * sstride], c3 = c[3 * sstride], c4 = c[4 * sstride], c5 = c[5 * sstride];
                    bool four = false;   // a solid cell among the six: the four-cell WENO3-Z stencil (weno_line_states, Schemes.cpp:815-831)
                    if (a.bc.solid)
#pragma unroll
                        for (int s6 = 0; s6 < 6; ++s6) four = four || Sf[base + s6 * sstride] != 0;
                    if (four) {
                        wl = weno3z(c1, c2, c3, a.weno_eps);
                        wr = weno3z(c4, c3, c2, a.weno_eps);
                    } else {
                        wl = weno5z(c0, c1, c2, c3, c4, a.weno_eps);
                        wr = weno5z(c5, c4, c3, c2, c1, a.weno_eps);
                    }
                }
                WL[q * S::NF + f] = wl;
                WR[q * S::NF + f] = wr;
            }
            __syncthreads();
        }
        // ---- 3. fluxes, written over the face values: slot f of WL is read and written by the thread of face f only
        const int na = n3[axis];
        const int lo_side = 2 * axis, hi_side = 2 * axis + 1;
        for (int f = tid; f < nF; f += NT) {
            const int f3[3] = {f % Fd[0], (f / Fd[0]) % Fd[1], f / (Fd[0] * Fd[1])};
            const int g3[3] = {o3[0] + f3[0], o3[1] + f3[1], o3[2] + f3[2]};
            bool inside = true;
#pragma unroll
            for (int d = 0; d < DIM; ++d) inside = inside && (d == axis ? g3[d] <= n3[d] : g3[d] < n3[d]);
            St<double, NV> F;
#pragma unroll
            for (int q = 0; q < NV; ++q) F[q] = 0.0;
            if (inside) {
                const int t = g3[axis];
                const bool lo_face = t == 0 && a.bc.halo[lo_side] == kHaloNone;
                const bool hi_face = t == na && a.bc.halo[hi_side] == kHaloNone;
                St<double, NV> UL, UR;
                if (lo_face || hi_face) {
                    int c3[3] = {g3[0], g3[1], g3[2]};
                    if (hi_face) c3[axis] = na - 1;
                    side_states<NV, FULL>(m, a.bc, a.eos, a.U, lo_face ? lo_side : hi_side, c3[0], c3[1], c3[2], UL, UR);
                    if constexpr (RECON != kFirstOrder) {
                        UL = round_trip(a.eos, UL);
                        UR = round_trip(a.eos, UR);
                    }
                } else if constexpr (RECON == kFirstOrder) {
                    // between two cells: the extended positions of the cells t-1 and t
                    const int base = (f3[2] * E[1] + f3[1]) * E[0] + f3[0];
#pragma unroll
                    for (int q = 0; q < NV; ++q) {
                        UL[q] = P[q * S::EXT + base];
                        UR[q] = P[q * S::EXT + base + sstride];
                    }
                } else {
                    int lc[3] = {g3[0], g3[1], g3[2]};
                    lc[axis] -= 1;
                    if (FULL && a.fb && (fb_flagged<DIM>(m, a.bc, a.fb, lc[0], lc[1], lc[2]) || fb_flagged<DIM>(m, a.bc, a.fb, g3[0], g3[1], g3[2]))) {
                        // next to a flagged cell: the two cells' states (the ghost of a side's halo beyond it)
                        UL = stencil_cons<DIM, NV>(m, a.bc, a.eos, a.U, lc[0], lc[1], lc[2]);
                        UR = stencil_cons<DIM, NV>(m, a.bc, a.eos, a.U, g3[0], g3[1], g3[2]);
                    } else {
                        St<double, NV> wl, wr;
#pragma unroll
                        for (int q = 0; q < NV; ++q) {
                            wl[q] = WL[q * S::NF + f];
                            wr[q] = WR[q * S::NF + f];
                        }
                        UL = p2c(a.eos, wl);
                        UR = p2c(a.eos, wr);
                    }
                }
                const double s = face_flux<RIEMANN>(a.eos, a.shock_blend, UL, UR, axis, F);
                if (s > smax) smax = s;
            }
#pragma unroll
            for (int q = 0; q < NV; ++q) WL[q * S::NF + f] = F[q];
        }
        __syncthreads();
        // ---- 4. balance of this axis
        const double A = m.area[axis];
        const double* Ff = WL;   // [NV][NF]
        for (int c = tid; c < NC; c += NT) {
            const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
            const int fl = (c3[2] * Fd[1] + c3[1]) * Fd[0] + c3[0];
            const int fr = fl + (axis == 0 ? 1 : (axis == 1 ? Fd[0] : Fd[0] * Fd[1]));
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                const double d = Ff[q * S::NF + fr] * A - Ff[q * S::NF + fl] * A;
                acc[q * NC + c] = axis == 0 ? 0.0 - d : acc[q * NC + c] - d;
            }
        }
        __syncthreads();
        }
}

// FULL = false: a run without part interfaces, non-reflecting sides, the positivity fallback or the body force (their
// code compiled out of the hot loop: a branch never taken still costs the others registers and instruction fetch).
// The epilogue's operands that no sweep reads (the tile's rows of U0 and of the viscous residual) head for L2 at the
// start of the tile, so that the epilogue's loads find them there; the arithmetic is untouched.
template <int NV, int TX, int TY, int TZ, int NT> __device__ __forceinline__ void prefetch_tile_rows(const StageArgs& a, const int o3[3]) {
    const bool u0 = a.mode == kCombine, rv = a.Rv != nullptr;
    if (!u0 && !rv) return;
    const Mesh& m = a.m;
    constexpr int R = TY * TZ;   // rows of TX cells
    for (int k = threadIdx.x; k < 2 * NV * R; k += NT) {
        const int which = k / (NV * R), q = (k / R) % NV, r = k % R;
        const int y = o3[1] + r % TY, z = o3[2] + r / TY;
        if (y >= m.ny || z >= m.nz) continue;
        const long long row = ((long long)z * m.ny + y) * m.nx + o3[0];
        if (which == 0 && u0) prefetch_l2(a.U0 + q * m.plane + row);
        if (which == 1 && rv) prefetch_l2(a.Rv + q * m.plane + row);
    }
}

template <int DIM, int RECON, int RIEMANN, int TX, int TY, int TZ, int NT, bool FULL = true>
__global__ void __launch_bounds__(NT) stage_kernel(const StageArgs a) {
    using S = StageShape<DIM, RECON, TX, TY, TZ>;
    constexpr int NV = S::NV, NC = S::NC;
    extern __shared__ double smem[];
    double* P = smem;                       // [NV][EXT]
    double* WL = P + S::P_SIZE;             // [NV][NF]
    double* WR = WL + NV * S::NF;           // [NV][NF]
    double* acc = WR + NV * S::NF;          // [NV][NC]
    double* red = acc + NV * NC;            // [32]
    unsigned char* Sf = reinterpret_cast<unsigned char*>(red + 32);   // [EXT]
    if (!*a.gate) return;

    const Mesh& m = a.m;
    const int tid = threadIdx.x;
    const int b = blockIdx.x + a.b0;
    const int t0 = b % a.tiles[0], t1 = (b / a.tiles[0]) % a.tiles[1], t2 = b / (a.tiles[0] * a.tiles[1]);
    const int o3[3] = {t0 * TX, t1 * TY, t2 * TZ};
    double smax = 0.0;
    prefetch_tile_rows<NV, TX, TY, TZ, NT>(a, o3);

    stage_axis<0, DIM, RECON, RIEMANN, TX, TY, TZ, NT, FULL>(a, P, WL, WR, acc, Sf, o3, smax);
    stage_axis<1, DIM, RECON, RIEMANN, TX, TY, TZ, NT, FULL>(a, P, WL, WR, acc, Sf, o3, smax);
    if constexpr (DIM == 3) stage_axis<2, DIM, RECON, RIEMANN, TX, TY, TZ, NT, FULL>(a, P, WL, WR, acc, Sf, o3, smax);
    // ---- epilogue: the residual and the stage update
    const double dt = a.ctl->dt;
    for (int c = tid; c < NC; c += NT) {
        const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
        const int g3[3] = {o3[0] + c3[0], o3[1] + c3[1], o3[2] + c3[2]};
        if (g3[0] >= m.nx || g3[1] >= m.ny || g3[2] >= m.nz) continue;
        const long long cell = ((long long)g3[2] * m.ny + g3[1]) * m.nx + g3[0];
        St<double, NV> r;
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            r[q] = acc[q * NC + c] * m.inv_cell;
            if (a.Rv) r[q] = r[q] + a.Rv[q * m.plane + cell];
        }
        // the body force, then the case's source terms, join after the viscous term (Simulation::assemble,
        // cpp/src/Simulation.cpp:1038-1049; RhsSourceTerms in the order Simulation::setup adds them, :372-412)
        if constexpr (FULL) {
            if (a.bc.grav_on) add_body_force<NV>(a.bc, read_state<NV>(a.bc, a.U, m.plane, cell), r);
            if (a.bc.src) add_source<NV>(a.bc, m.plane, cell, r);
        }
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const long long e = q * m.plane + cell;
            double o;
            if (a.mode == kStoreR)
                o = r[q];
            else if (a.mode == kAxpy)
                o = a.U[e] + dt * r[q];
            else
                o = a.ca * a.U0[e] + a.cb * (a.U[e] + dt * r[q]);
            a.out[e] = o;
        }
    }
    const double bm = block_max<NT>(smax, red);
    if (tid == 0) a.blockmax[b] = bm;
}

}   // namespace fvg
