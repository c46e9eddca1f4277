// The mixed-precision form of the stage and viscous kernels: stencil, flux and viscous arithmetic in FP32, the
// conserved state and its Runge-Kutta accumulation in FP64.
//
// What stays FP64: the state in HBM and every stage update (a U0 + b (U + dt R), with R widened to double), and the
// pressure recovery p = (gamma - 1)(E - 1/2 rho |u|^2) of every cell (cons_to_prim in double when a cell is loaded, so a
// low-Mach cell, where E and the kinetic energy nearly cancel, loses nothing). What runs in FP32 (compiled with fast
// single-precision division and square root, and contraction into FMAs): the WENO-Z / MUSCL reconstruction of the
// primitives, the Riemann solver, the flux balance, the viscous stresses and heat flux. The linear and WENO5-Z face values,
// the balance and the FP64 update round every operation explicitly instead, so that every kernel that solves a face or
// updates a cell (the per-axis sweep, the cross form, the batched kernels) gives it the same bits.
//
// One algorithmic difference from the plain form: the Riemann solver takes the reconstructed primitive states directly
// (their density and pressure floored as cons_to_prim floors them) instead of converting them to conservative form and
// back, which in FP32 would recover the face pressure from a difference of nearly equal numbers. In exact arithmetic the
// two are the same; the tests state the L1 / Linf distance of this form from the FP64 oracle per field and per case.
#pragma once

#include <type_traits>

#include "grid.cuh"
#include "stage.cuh"
#include "tma.cuh"
#include "viscous.cuh"

namespace fvg {

// HLLC / low-Mach HLLC of a face from its two primitive states (the Riemann solver of the mixed form)
template <int RIEMANN, int NV>
__device__ __forceinline__ float face_flux_prim(const Eos<float>& e, float shock_blend, St<float, NV> WL, St<float, NV> WR, int axis, St<float, NV>& F) {
    WL[0] = vmax(WL[0], Num<float>::eos_eps);
    WL[3] = vmax(WL[3], Num<float>::eos_eps);
    WR[0] = vmax(WR[0], Num<float>::eos_eps);
    WR[3] = vmax(WR[3], Num<float>::eos_eps);
    const float inv_L = 1.0f / WL[0], inv_R = 1.0f / WR[0];
    const float c_L = sound_speed_inv(e, WL[3], inv_L), c_R = sound_speed_inv(e, WR[3], inv_R);
    if constexpr (RIEMANN == kLowMach) {
        float mL2 = WL[1] * WL[1] + WL[2] * WL[2], mR2 = WR[1] * WR[1] + WR[2] * WR[2];
        if constexpr (NV == 5) {
            mL2 += WL[4] * WL[4];
            mR2 += WR[4] * WR[4];
        }
        const float M_L = sqrtf(mL2) / (c_L + Num<float>::mach_eps);
        const float M_R = sqrtf(mR2) / (c_R + Num<float>::mach_eps);
        const float z = vmin(vmax(vmax(M_L, M_R), 1e-4f), 1.0f);
#pragma unroll
        for (int a = 0; a < (NV == 5 ? 3 : 2); ++a) {
            const int m = a == 0 ? 1 : (a == 1 ? 2 : 4);
            const float avg = 0.5f * (WL[m] + WR[m]);
            const float half = 0.5f * (WL[m] - WR[m]);
            WL[m] = avg + z * half;
            WR[m] = avg - z * half;
        }
    }
    return hllc_core(WL, WR, p2c(e, WL), p2c(e, WR), inv_L, inv_R, c_L, c_R, axis, shock_blend, F);
}

// the fifth-order upwind value right of c2 from c0 .. c4: 0.1 p0 + 0.6 p1 + 0.3 p2 of the three candidate stencils
// (explicitly rounded FMAs, as the single-precision weno5z: the same bits in every kernel)
__device__ __forceinline__ float lin5(float c0, float c1, float c2, float c3, float c4) {
    const float s = __fmaf_rn(-3.0f, c4, __fmaf_rn(27.0f, c3, __fmaf_rn(47.0f, c2, __fmaf_rn(-13.0f, c1, __fmul_rn(2.0f, c0)))));
    return __fmul_rn(s, 1.0f / 60.0f);
}

template <int DIM, int RECON, int TX, int TY, int TZ> struct MixedShape {
    static constexpr int NV = DIM == 3 ? 5 : 4;
    static constexpr int H = RECON == kWeno5 ? 3 : 2;
    static constexpr int NC = TX * TY * TZ;
    static constexpr int T3[3] = {TX, TY, TZ};
    static constexpr int ext(int a) { return (T3[0] + (a == 0 ? 2 * H : 0)) * (T3[1] + (a == 1 ? 2 * H : 0)) * (T3[2] + (a == 2 ? 2 * H : 0)); }
    static constexpr int nf(int a) { return (T3[0] + (a == 0)) * (T3[1] + (a == 1)) * (T3[2] + (a == 2)); }
    static constexpr int cmax(int a, int b) { return a > b ? a : b; }
    static constexpr int EXT = cmax(cmax(ext(0), ext(1)), DIM == 3 ? ext(2) : 0);
    static constexpr int NF = cmax(cmax(nf(0), nf(1)), DIM == 3 ? nf(2) : 0);
    // floats: P [NV][EXT], WL / WR [NV][NF] (the fluxes overwrite WL), acc [NV][NC], 64 for the reduction
    static constexpr int SMEM_FLOATS = NV * EXT + 2 * NV * NF + NV * NC + 64;
    static constexpr int FLAG_BYTES = (EXT + 7) / 8 * 8;   // solidity of the extended tile (WENO5-Z beside an immersed body)
    static constexpr size_t SMEM_BYTES = sizeof(float) * SMEM_FLOATS + FLAG_BYTES;
};

// One axis of the tile sweep of mixed_stage_kernel (compile-time extents).
// GATED (WENO5-Z with the learned sensor): the tile's flag for this axis (one byte per tile and axis, from the sensor's
// last refresh) makes the reconstructions of the sweep linear (0) or WENO5-Z (1), a branch uniform over the CTA; the seam
// faces of a linear tile whose tile across stays WENO5-Z take WENO5-Z in a short pass of their own.
// TMA (mixed_stage_kernel_tma): a tile whose box lies inside the mesh is staged by one bulk tensor copy into the face-value
// arrays (free during the load) and converted from there; the others take the index-mapping loader. `phase` counts the
// barrier's completed copies (its parity is the one to wait for).
template <int AXIS, int DIM, int RECON, int RIEMANN, int TX, int TY, int TZ, int NT, bool GATED = false, bool FULL = true, bool TMA = false>
__device__ __forceinline__ void mixed_axis(const StageArgs& a, const Eos<float>& ef, float sb, float weps, float* __restrict__ P,
                                           float* __restrict__ WL, float* __restrict__ WR, float* __restrict__ acc, unsigned char* __restrict__ Sf,
                                           const int o3[3], float& smax, const CUtensorMap* maps = nullptr, unsigned long long* bar = nullptr,
                                           unsigned* phase = nullptr) {
    using S = MixedShape<DIM, RECON, TX, TY, TZ>;
    constexpr int NV = S::NV, H = S::H, NC = S::NC;
    constexpr int axis = AXIS;
    const Mesh& m = a.m;
    const int tid = threadIdx.x;
    const int n3[3] = {m.nx, m.ny, m.nz};
    {
        constexpr int E[3] = {TX + (AXIS == 0 ? 2 * H : 0), TY + (AXIS == 1 ? 2 * H : 0), TZ + (AXIS == 2 ? 2 * H : 0)};
        constexpr int Fd[3] = {TX + (AXIS == 0), TY + (AXIS == 1), TZ + (AXIS == 2)};
        constexpr int nE = E[0] * E[1] * E[2], nF = Fd[0] * Fd[1] * Fd[2];
        // ---- 1. load: the primitive state recovered in FP64, stored as FP32
        bool via_tma = false;
        if constexpr (TMA) {
            constexpr int BX = AXIS == 0 ? 16 : TX, BY = TY + (AXIS == 1 ? 2 * H : 0), BZ = TZ + (AXIS == 2 ? 2 * H : 0);
            const int x0 = AXIS == 0 ? o3[0] - 4 : o3[0], y0 = AXIS == 1 ? o3[1] - H : o3[1], z0 = AXIS == 2 ? o3[2] - H : o3[2];
            via_tma = x0 >= 0 && x0 + BX <= n3[0] && y0 >= 0 && y0 + BY <= n3[1] && z0 >= 0 && z0 + BZ <= n3[2] && (tma::su32(WL) & 127u) == 0;
            if (via_tma) {
                const double* stg = reinterpret_cast<const double*>(WL);
                if (tid == 0) {
                    tma::fence_proxy_async();
                    tma::mbar_expect_tx(bar, (unsigned)(BX * BY * BZ * NV * 8));
                    tma::load_4d(WL, &maps[AXIS], x0, y0, z0, 0, bar);
                }
                // every thread waits for this copy's phase of the barrier, at most 2^22 polls; a copy that never
                // completes stops the run (status 5) instead of hanging the GPU
                bool done = false;
                for (int it = 0; it < (1 << 22) && !done; ++it) done = tma::mbar_try_wait(bar, *phase & 1u);
                ++*phase;
                if (!done && tid == 0) atomicExch(const_cast<int*>(&a.ctl->status), 5);
                for (int e = tid; e < nE; e += NT) {
                    const int l3[3] = {e % E[0], (e / E[0]) % E[1], e / (E[0] * E[1])};
                    const int si = (l3[2] * BY + l3[1]) * BX + (AXIS == 0 ? l3[0] + 1 : l3[0]);
                    St<double, NV> u;
#pragma unroll
                    for (int q = 0; q < NV; ++q) u[q] = done ? stg[q * (BX * BY * BZ) + si] : 1.0;
                    const St<double, NV> w = c2p(a.eos, u);
#pragma unroll
                    for (int q = 0; q < NV; ++q) P[q * S::EXT + e] = (float)w[q];
                }
            }
        }
        if (!via_tma)
        for (int e = tid; e < nE; e += NT) {
            int l3[3] = {e % E[0], (e / E[0]) % E[1], e / (E[0] * E[1])};
            l3[axis] -= H;
            const St<double, NV> w = c2p(a.eos, stencil_cons<DIM, NV, FULL>(m, a.bc, a.eos, a.U, o3[0] + l3[0], o3[1] + l3[1], o3[2] + l3[2]));
            if constexpr (RECON == kWeno5)
                if (!TMA && a.bc.solid) Sf[e] = stencil_solid<DIM>(m, a.bc, o3[0] + l3[0], o3[1] + l3[1], o3[2] + l3[2]);
#pragma unroll
            for (int q = 0; q < NV; ++q) P[q * S::EXT + e] = (float)w[q];
        }
        __syncthreads();
        const int sstride = axis == 0 ? 1 : (axis == 1 ? E[0] : E[0] * E[1]);
        // GATED: whether this tile's reconstructions along the axis are linear, and whether each of its two seam faces
        // along the axis (shared with the tile before and the tile after, which solve them too) may be: only when the
        // tile across is linear as well, so both tiles compute the same flux there and the balance stays conservative.
        // A seam face is the tile's first face and its last face inside the mesh (a partial last tile included); on a
        // periodic axis the neighbour of an end tile is the other end tile; beyond any other side no tile solves the
        // face twice (and the gate keeps such tiles WENO5-Z).
        bool tile_linear = false, seam_lo = false, seam_hi = false;
        int hi_face = 0;
        if constexpr (GATED) {
            const unsigned char* fl = a.sens_flags + (long long)AXIS * a.tiles[0] * a.tiles[1] * a.tiles[2];
            const int b = blockIdx.x + a.b0;
            tile_linear = fl[b] == 0;
            if (tile_linear) {
                const int nt = a.tiles[AXIS];
                const int st = AXIS == 0 ? 1 : (AXIS == 1 ? a.tiles[0] : a.tiles[0] * a.tiles[1]);
                const int ta = AXIS == 0 ? b % a.tiles[0] : (AXIS == 1 ? (b / a.tiles[0]) % a.tiles[1] : b / (a.tiles[0] * a.tiles[1]));
                const bool wrap_lo = a.bc.halo[2 * AXIS] == kHaloWrap, wrap_hi = a.bc.halo[2 * AXIS + 1] == kHaloWrap;
                seam_lo = ta > 0 ? fl[b - st] == 0 : (wrap_lo ? fl[b + (nt - 1) * st] == 0 : true);
                seam_hi = ta < nt - 1 ? fl[b + st] == 0 : (wrap_hi ? fl[b - (nt - 1) * st] == 0 : true);
            }
            hi_face = n3[AXIS] - o3[AXIS] < Fd[AXIS] - 1 ? n3[AXIS] - o3[AXIS] : Fd[AXIS] - 1;
        }
        // ---- 2. face values
        for (int it = tid; it < nF * NV; it += NT) {
            const int f = it % nF, q = it / nF;
            const int f3[3] = {f % Fd[0], (f / Fd[0]) % Fd[1], f / (Fd[0] * Fd[1])};
            const float* c = P + q * S::EXT + (f3[2] * E[1] + f3[1]) * E[0] + f3[0];
            float wl, wr;
            if constexpr (RECON == kMuscl) {
                const float c0 = c[0], c1 = c[sstride], c2 = c[2 * sstride], c3 = c[3 * sstride];
                const float bb = c2 - c1;
                wl = c1 + 0.5f * limiter(a.limiter, c1 - c0, bb);
                wr = c2 - 0.5f * limiter(a.limiter, c3 - c2, bb);
            } else if constexpr (RECON == kWeno3) {
                wl = weno3z(c[0], c[sstride], c[2 * sstride], weps);
                wr = weno3z(c[3 * sstride], c[2 * sstride], c[sstride], weps);
            } else {
                const float c0 = c[0], c1 = c[sstride], c2 = c[2 * sstride], c3 = c[3 * sstride], c4 = c[4 * sstride], c5 = c[5 * sstride];
                const int base = (f3[2] * E[1] + f3[1]) * E[0] + f3[0];
                bool four = false;
                if (!TMA && a.bc.solid)   // (the TMA kernel never runs with an immersed body)
#pragma unroll
                    for (int s6 = 0; s6 < 6; ++s6) four = four || Sf[base + s6 * sstride] != 0;
                if (four) {
                    wl = weno3z(c1, c2, c3, weps);
                    wr = weno3z(c4, c3, c2, weps);
                } else if (tile_linear) {
                    // a seam face whose tile across stays WENO5-Z is left to the seam pass below (so that this pass's
                    // warps all take the cheap branch)
                    if (!(f3[AXIS] == 0 ? seam_lo : (f3[AXIS] == hi_face ? seam_hi : true))) continue;
                    // linear fifth-order upwind values where the sensor passed the tile (the WENO-Z weights at their
                    // linear values 0.1, 0.6, 0.3)
                    wl = lin5(c0, c1, c2, c3, c4);
                    wr = lin5(c5, c4, c3, c2, c1);
                } else {
                    wl = weno5z(c0, c1, c2, c3, c4, weps);
                    wr = weno5z(c5, c4, c3, c2, c1, weps);
                }
            }
            WL[q * S::NF + f] = wl;
            WR[q * S::NF + f] = wr;
        }
        if constexpr (GATED) {
            // the seam pass: a linear tile's seam faces whose tile across stays WENO5-Z take WENO5-Z, as that tile does
            if (tile_linear && (!seam_lo || !seam_hi)) {
                constexpr int PL = nF / Fd[AXIS];   // faces of one layer across the axis
                const int layers = (!seam_lo ? 1 : 0) + (!seam_hi ? 1 : 0);
                for (int it = tid; it < layers * PL * NV; it += NT) {
                    const int q = it / (layers * PL), rem = it % (layers * PL), layer = rem / PL, r = rem % PL;
                    int f3[3];
                    f3[AXIS] = (layer == 0 && !seam_lo) ? 0 : hi_face;
                    constexpr int A1 = AXIS == 0 ? 1 : 0, A2 = AXIS == 2 ? 1 : 2;
                    f3[A1] = r % Fd[A1];
                    f3[A2] = r / Fd[A1];
                    const int f = (f3[2] * Fd[1] + f3[1]) * Fd[0] + f3[0];
                    const int base = (f3[2] * E[1] + f3[1]) * E[0] + f3[0];
                    const float* c = P + q * S::EXT + base;
                    const float c0 = c[0], c1 = c[sstride], c2 = c[2 * sstride], c3 = c[3 * sstride], c4 = c[4 * sstride], c5 = c[5 * sstride];
                    bool four = false;
                    if (!TMA && a.bc.solid)   // (the TMA kernel never runs with an immersed body)
#pragma unroll
                        for (int s6 = 0; s6 < 6; ++s6) four = four || Sf[base + s6 * sstride] != 0;
                    float wl, wr;
                    if (four) {
                        wl = weno3z(c1, c2, c3, weps);
                        wr = weno3z(c4, c3, c2, weps);
                    } else {
                        wl = weno5z(c0, c1, c2, c3, c4, weps);
                        wr = weno5z(c5, c4, c3, c2, c1, weps);
                    }
                    WL[q * S::NF + f] = wl;
                    WR[q * S::NF + f] = wr;
                }
            }
        }
        __syncthreads();
        // ---- 3. fluxes
        const int na = n3[axis], lo_side = 2 * axis, hi_side = 2 * axis + 1;
        for (int f = tid; f < nF; f += NT) {
            const int f3[3] = {f % Fd[0], (f / Fd[0]) % Fd[1], f / (Fd[0] * Fd[1])};
            const int g3[3] = {o3[0] + f3[0], o3[1] + f3[1], o3[2] + f3[2]};
            bool inside = true;
#pragma unroll
            for (int d = 0; d < DIM; ++d) inside = inside && (d == axis ? g3[d] <= n3[d] : g3[d] < n3[d]);
            St<float, NV> F;
#pragma unroll
            for (int q = 0; q < NV; ++q) F[q] = 0.0f;
            if (inside) {
                const int t = g3[axis];
                const bool lo_face = t == 0 && a.bc.halo[lo_side] == kHaloNone;
                const bool hi_face = t == na && a.bc.halo[hi_side] == kHaloNone;
                St<float, NV> wl, wr;
                if (lo_face || hi_face) {
                    int c3[3] = {g3[0], g3[1], g3[2]};
                    if (hi_face) c3[axis] = na - 1;
                    St<double, NV> UL, UR;
                    side_states<NV, FULL>(m, a.bc, a.eos, a.U, lo_face ? lo_side : hi_side, c3[0], c3[1], c3[2], UL, UR);
                    const St<double, NV> dl = c2p(a.eos, UL), dr = c2p(a.eos, UR);
#pragma unroll
                    for (int q = 0; q < NV; ++q) {
                        wl[q] = (float)dl[q];
                        wr[q] = (float)dr[q];
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < NV; ++q) {
                        wl[q] = WL[q * S::NF + f];
                        wr[q] = WR[q * S::NF + f];
                    }
                }
                const float s = face_flux_prim<RIEMANN>(ef, sb, wl, wr, axis, F);
                if (s > smax) smax = s;
            }
#pragma unroll
            for (int q = 0; q < NV; ++q) WL[q * S::NF + f] = F[q];
        }
        __syncthreads();
        // ---- 4. balance of this axis
        const float A = (float)m.area[axis];
        for (int c = tid; c < NC; c += NT) {
            const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
            const int fl = (c3[2] * Fd[1] + c3[1]) * Fd[0] + c3[0];
            const int fr = fl + (axis == 0 ? 1 : (axis == 1 ? Fd[0] : Fd[0] * Fd[1]));
#pragma unroll
            for (int q = 0; q < NV; ++q) {   // (explicit FMAs, never left to the compiler: every kernel of the mixed
                                               // form sums a cell's balance to the same bits)
                const float df = WL[q * S::NF + fr] - WL[q * S::NF + fl];
                acc[q * NC + c] = axis == 0 ? -__fmul_rn(df, A) : __fmaf_rn(-df, A, acc[q * NC + c]);
            }
        }
        __syncthreads();
        }
}

// The epilogue of the mixed form. A cell's global operands (U, U0, the viscous residual) are loaded first, all variables
// at once, so that their latency overlaps; then every FP64 operation is an explicit intrinsic, FMAs placed by hand
// (nothing left for a compiler pass to contract one way in one kernel and another way in the next: each kernel that
// updates a cell gives it the same bits).
template <int NV> struct CellIn {
    double u[NV], u0[NV], rv[NV];
};
template <int NV> __device__ __forceinline__ void cell_load(const StageArgs& a, long long cell, CellIn<NV>& in) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        const long long e = q * a.m.plane + cell;
        in.u[q] = a.mode != kStoreR ? a.U[e] : 0.0;
        in.u0[q] = a.mode == kCombine ? a.U0[e] : 0.0;
        in.rv[q] = a.Rvf ? (q == 0 ? 0.0 : (double)a.Rvf[(q - 1) * a.m.plane + cell]) : (a.Rv ? a.Rv[e] : 0.0);
    }
}
// variable q's output from the tile's FP32 balance sum: the residual sum / volume plus the viscous residual (Rv, or the
// 3-D FP32 viscous balance sum of Rvf / volume; the density's viscous term is +0), then R, U + dt R, or ca U0 + cb (U + dt R)
template <int NV> __device__ __forceinline__ double cell_out(const StageArgs& a, const CellIn<NV>& in, int q, float sum, double dt) {
    double r = __dmul_rn((double)sum, a.m.inv_cell);
    if (a.Rvf)
        r = q == 0 ? __dadd_rn(r, 0.0) : __fma_rn(in.rv[q], a.m.inv_cell, r);
    else if (a.Rv)
        r = __dadd_rn(r, in.rv[q]);
    if (a.mode == kStoreR) return r;
    const double u = __fma_rn(dt, r, in.u[q]);
    if (a.mode == kAxpy) return u;
    return __fma_rn(a.ca, in.u0[q], __dmul_rn(a.cb, u));
}

// The mixed-precision stage kernel: the tile sweep of stage_kernel (same phases, same launch geometry) with FP32 stencil
// arithmetic; see the file comment for what stays FP64.
// FULL = false: a run without part interfaces or non-reflecting sides (their code compiled out of the hot loop)
template <int DIM, int RECON, int RIEMANN, int TX, int TY, int TZ, int NT, bool GATED = false, bool FULL = true>
__global__ void __launch_bounds__(NT) mixed_stage_kernel(const StageArgs a) {
    using S = MixedShape<DIM, RECON, TX, TY, TZ>;
    constexpr int NV = S::NV, NC = S::NC;
    extern __shared__ double smem_d[];
    double* red = smem_d;                                      // [32]
    float* P = reinterpret_cast<float*>(smem_d + 32);         // [NV][EXT]
    float* WL = P + NV * S::EXT;                               // [NV][NF]
    float* WR = WL + NV * S::NF;                               // [NV][NF]
    float* acc = WR + NV * S::NF;                              // [NV][NC]
    unsigned char* Sf = reinterpret_cast<unsigned char*>(acc + NV * NC);   // [EXT]
    if (!*a.gate) return;
    const Mesh& m = a.m;
    const Eos<float> ef{a.eos.type, (float)a.eos.gamma, (float)a.eos.p_inf};
    const float sb = (float)a.shock_blend, weps = (float)a.weno_eps;
    const int tid = threadIdx.x, b = blockIdx.x + a.b0;
    const int o3[3] = {(b % a.tiles[0]) * TX, ((b / a.tiles[0]) % a.tiles[1]) * TY, (b / (a.tiles[0] * a.tiles[1])) * TZ};
    float smax = 0.0f;
    mixed_axis<0, DIM, RECON, RIEMANN, TX, TY, TZ, NT, GATED, FULL>(a, ef, sb, weps, P, WL, WR, acc, Sf, o3, smax);
    mixed_axis<1, DIM, RECON, RIEMANN, TX, TY, TZ, NT, GATED, FULL>(a, ef, sb, weps, P, WL, WR, acc, Sf, o3, smax);
    if constexpr (DIM == 3) mixed_axis<2, DIM, RECON, RIEMANN, TX, TY, TZ, NT, GATED, FULL>(a, ef, sb, weps, P, WL, WR, acc, Sf, o3, smax);
    // ---- epilogue: the residual widened to FP64 and the FP64 stage update
    const double dt = a.ctl->dt;
    for (int c = tid; c < NC; c += NT) {
        const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
        const int g3[3] = {o3[0] + c3[0], o3[1] + c3[1], o3[2] + c3[2]};
        if (g3[0] >= m.nx || g3[1] >= m.ny || g3[2] >= m.nz) continue;
        const long long cell = ((long long)g3[2] * m.ny + g3[1]) * m.nx + g3[0];
        CellIn<NV> in;
        cell_load(a, cell, in);
#pragma unroll
        for (int q = 0; q < NV; ++q) a.out[q * m.plane + cell] = cell_out(a, in, q, acc[q * NC + c], dt);
    }
    const double bm = block_max<NT>((double)smax, red);
    if (tid == 0) a.blockmax[b] = bm;
}

template <int TX, int TY, int TZ> struct MixedViscShape {
    static constexpr int NC = TX * TY * TZ;
    // red [32 doubles], then float4 arrays: V [NB] box (u, v, w, T), G [NE] (the sweep's four gradient entries), F [NF]
    // (the four face fluxes: rho u, rho v, rho E, rho w; the mass flux is 0), acc [NC] (the four balances); then R [NB]
    // floats (the box's rho): 4 CTAs of the 8x8x8 tile fit on an SM
    static constexpr int BX = TX + 2, BY = TY + 2, BZ = TZ + 2, NB = BX * BY * BZ;
    static constexpr int cmax(int x, int y) { return x > y ? x : y; }
    static constexpr int NE = cmax(cmax((TX + 2) * TY * TZ, TX * (TY + 2) * TZ), TX * TY * (TZ + 2));
    static constexpr int NF = cmax(cmax((TX + 1) * TY * TZ, TX * (TY + 1) * TZ), TX * TY * (TZ + 1));
    static constexpr size_t SMEM_BYTES = 256 + 16 * (NB + NE + NF + NC) + 4 * NB;
};
// component a (0 u, 1 v, 2 w, 3 T) of a box position's float4
__device__ __forceinline__ float f4c(float4 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : (a == 2 ? v.z : v.w)); }
// The mixed-precision viscous kernel: viscous_kernel's phases in FP32; the padded state is read in FP64 and each box
// position's velocity and T = p / rho come from an FP64 pressure recovery. The velocity gradients
// G[a][b] = (d(rho u_a)/dx_b - u_a d(rho)/dx_b) / rho take the box's rho and u_a: (rho+ (u_a+ - u_a) - rho- (u_a- - u_a))
// / (2 h_b rho), the same difference in exact arithmetic. A tile none of whose sides is a wall, inlet or outlet (only
// periodic sides and part interfaces around it) reads its box without the ghost rules and solves its faces without the
// wall tests; a tile wholly inside the mesh skips the test for faces beyond it. The four values a position, a face or a
// cell carries sit together in one float4 (one shared-memory access each); each axis's balance shares a phase with the
// next axis's gradients (six barriers per tile); WALLS = false drops the ghost rules and wall tests from launches whose
// every side is periodic or a part interface. Measured at 256^3 (Taylor-Green): 0.77 ms per launch against 1.14 ms for
// the first form (rho u_a in the box, 1 / rho, the general path for every tile), the same distance from the FP64 viscous
// residual (1.24e-3 of its largest value, both).
template <int TX, int TY, int TZ, int NT, bool WALLS = true>
__global__ void __launch_bounds__(NT, 4) mixed_viscous_kernel(const ViscArgs a) {
    using S = MixedViscShape<TX, TY, TZ>;
    constexpr int NC = S::NC, BX = S::BX, BY = S::BY, NB = S::NB;
    extern __shared__ double smem_d[];
    double* red = smem_d;
    float4* V = reinterpret_cast<float4*>(smem_d + 32);   // [NB]: u, v, w, T
    float4* G = V + NB;
    float4* Fv = G + S::NE;
    float4* acc = Fv + S::NF;
    float* R = reinterpret_cast<float*>(acc + NC);         // [NB]: rho
    if (!*a.gate) return;
    const Mesh& m = a.m;
    const int tid = threadIdx.x, b = blockIdx.x + a.b0;
    const int o3[3] = {(b % a.tiles[0]) * TX, ((b / a.tiles[0]) % a.tiles[1]) * TY, (b / (a.tiles[0] * a.tiles[1])) * TZ};
    const int n3[3] = {m.nx, m.ny, m.nz};
    const float h[3] = {(float)m.dx, (float)m.dy, (float)m.dz};
    const float mu = (float)a.mu, kc = (float)a.k_cond;
    constexpr int GA[3][4] = {{0, 1, 2, 0}, {0, 1, 2, 1}, {0, 1, 2, 2}};
    constexpr int GB[3][4] = {{1, 1, 2, 2}, {0, 0, 2, 2}, {0, 1, 0, 1}};
    auto bidx = [&](int i, int j, int k) { return ((k + 1) * BY + (j + 1)) * BX + (i + 1); };
    // whether a side of the tile lies on a side of the mesh that is neither periodic nor a part interface
    bool walls = false;
    if constexpr (WALLS) {
#pragma unroll
        for (int x = 0; x < 3; ++x) walls = walls || (o3[x] == 0 && !a.through[2 * x]) || (o3[x] + (x == 0 ? TX : (x == 1 ? TY : TZ)) >= n3[x] && !a.through[2 * x + 1]);
    }
    const bool full = o3[0] + TX <= n3[0] && o3[1] + TY <= n3[1] && o3[2] + TZ <= n3[2];   // no cell of the tile beyond the mesh
    for (int e = tid; e < NB; e += NT) {
        int g[3] = {o3[0] + e % BX - 1, o3[1] + (e / BX) % BY - 1, o3[2] + e / (BX * BY) - 1};
#pragma unroll
        for (int x = 0; x < 3; ++x)
            if (a.periodic[x] && (g[x] < 0 || g[x] >= n3[x])) g[x] = ((g[x] % n3[x]) + n3[x]) % n3[x];
#pragma unroll
        for (int x = 0; x < 3; ++x) g[x] = box_clamp(a, x, g[x], n3[x]);
        St<double, 5> u;
        if constexpr (WALLS)
            u = walls ? padded_cons(a, g[0], g[1], g[2]) : cell_at(a, g[0], g[1], g[2]);
        else
            u = cell_at(a, g[0], g[1], g[2]);
        double inv;
        const St<double, 5> w = c2p(a.eos, u, inv);
        R[e] = (float)u[0];
        V[e] = make_float4((float)w[1], (float)w[2], (float)w[4], (float)(w[3] * inv));
    }
    __syncthreads();
    auto sweep = [&](auto axis_c) {
        constexpr int d = decltype(axis_c)::value;
        constexpr int E[3] = {TX + (d == 0 ? 2 : 0), TY + (d == 1 ? 2 : 0), TZ + (d == 2 ? 2 : 0)};
        constexpr int Fd[3] = {TX + (d == 0), TY + (d == 1), TZ + (d == 2)};
        constexpr int nE = E[0] * E[1] * E[2], nF = Fd[0] * Fd[1] * Fd[2];
        // the axes b of this sweep's four entries: GB[d][0..3] takes two distinct values, b0 and b1
        constexpr int b0 = GB[d][0], b1 = GB[d][1] != GB[d][0] ? GB[d][1] : GB[d][2];
        constexpr int off0 = b0 == 0 ? 1 : (b0 == 1 ? BX : BX * BY), off1 = b1 == 0 ? 1 : (b1 == 1 ? BX : BX * BY);
        for (int e = tid; e < nE; e += NT) {
            int l[3] = {e % E[0], (e / E[0]) % E[1], e / (E[0] * E[1])};
            l[d] -= 1;
            const int p = bidx(l[0], l[1], l[2]);
            const float rc = R[p];
            const float inv_rho = 1.0f / vmax(rc, Num<float>::eos_eps);
            const float rp0 = R[p + off0], rm0 = R[p - off0], rp1 = R[p + off1], rm1 = R[p - off1];
            const float4 vc = V[p], vp0 = V[p + off0], vm0 = V[p - off0], vp1 = V[p + off1], vm1 = V[p - off1];
            const float i20 = 0.5f / h[b0], i21 = 0.5f / h[b1];
            float gs[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int ga = GA[d][s];
                const bool first = GB[d][s] == b0;
                const float uc = f4c(vc, ga);
                const float up = first ? f4c(vp0, ga) : f4c(vp1, ga), um = first ? f4c(vm0, ga) : f4c(vm1, ga);
                const float rp = first ? rp0 : rp1, rm = first ? rm0 : rm1;
                gs[s] = (rp * (up - uc) - rm * (um - uc)) * (first ? i20 : i21) * inv_rho;
            }
            G[e] = make_float4(gs[0], gs[1], gs[2], gs[3]);
        }
        __syncthreads();
        const float area = (float)m.area[d];
        const float inv_h = 1.0f / h[d];
        constexpr int estride = d == 0 ? 1 : (d == 1 ? E[0] : E[0] * E[1]);
        constexpr int bstride = d == 0 ? 1 : (d == 1 ? BX : BX * BY);
        for (int f = tid; f < nF; f += NT) {
            const int f3[3] = {f % Fd[0], (f / Fd[0]) % Fd[1], f / (Fd[0] * Fd[1])};
            const int eL = (f3[2] * E[1] + f3[1]) * E[0] + f3[0];
            const int eR = eL + estride;
            int lc[3] = {f3[0], f3[1], f3[2]};
            lc[d] -= 1;
            const int pL = bidx(lc[0], lc[1], lc[2]), pR = pL + bstride;
            float out[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            bool inside = true;
            int xL = eL, xR = eR;
            bool phys = false, lo = false;
            if (WALLS && walls) {
                const int g3[3] = {o3[0] + f3[0], o3[1] + f3[1], o3[2] + f3[2]};
#pragma unroll
                for (int x = 0; x < 3; ++x) inside = inside && (x == d ? g3[x] <= n3[x] : g3[x] < n3[x]);
                const int t = g3[d];
                lo = t == 0;
                const bool hi = t == n3[d];
                const bool lo_wall = lo && !a.through[2 * d], hi_wall = hi && !a.through[2 * d + 1];
                xL = lo_wall ? eR : eL;
                xR = hi_wall ? eL : eR;
                phys = a.bface2 && (lo_wall || hi_wall);
            } else if (!full) {
                const int g3[3] = {o3[0] + f3[0], o3[1] + f3[1], o3[2] + f3[2]};
#pragma unroll
                for (int x = 0; x < 3; ++x) inside = inside && (x == d ? g3[x] <= n3[x] : g3[x] < n3[x]);
            }
            if (inside) {
                float Gc[4];
                if (WALLS && phys) {
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        const int ga = GA[d][s], gb = GB[d][s];
                        const int pg = lo ? pL : pR, pc = lo ? pR : pL;
                        const int off = gb == 0 ? 1 : (gb == 1 ? BX : BX * BY);
                        const float fp = 0.5f * (f4c(V[pg + off], ga) + f4c(V[pc + off], ga));
                        const float fm = 0.5f * (f4c(V[pg - off], ga) + f4c(V[pc - off], ga));
                        Gc[s] = (fp - fm) * (0.5f / h[gb]);
                    }
                } else {
                    const float4 gl = G[xL], gr = G[xR];
                    Gc[0] = 0.5f * (gl.x + gr.x);
                    Gc[1] = 0.5f * (gl.y + gr.y);
                    Gc[2] = 0.5f * (gl.z + gr.z);
                    Gc[3] = 0.5f * (gl.w + gr.w);
                }
                const float4 vl = V[pL], vr = V[pR];
                float Gn[3], vf[3];
#pragma unroll
                for (int x = 0; x < 3; ++x) {
                    Gn[x] = (f4c(vr, x) - f4c(vl, x)) * inv_h;
                    vf[x] = 0.5f * (f4c(vl, x) + f4c(vr, x));
                }
                const float dT = (vr.w - vl.w) * inv_h;
                float tau[3];
                if (d == 0) {
                    tau[0] = mu * ((4.0f / 3.0f) * Gn[0] - (2.0f / 3.0f) * (Gc[1] + Gc[2]));
                    tau[1] = mu * (Gn[1] + Gc[0]);
                    tau[2] = mu * (Gn[2] + Gc[3]);
                } else if (d == 1) {
                    tau[0] = mu * (Gn[0] + Gc[1]);
                    tau[1] = mu * ((4.0f / 3.0f) * Gn[1] - (2.0f / 3.0f) * (Gc[0] + Gc[2]));
                    tau[2] = mu * (Gn[2] + Gc[3]);
                } else {
                    tau[0] = mu * (Gn[0] + Gc[2]);
                    tau[1] = mu * (Gn[1] + Gc[3]);
                    tau[2] = mu * ((4.0f / 3.0f) * Gn[2] - (2.0f / 3.0f) * (Gc[0] + Gc[1]));
                }
                out[0] = tau[0] * area;
                out[1] = tau[1] * area;
                out[2] = (vf[0] * tau[0] + vf[1] * tau[1] + vf[2] * tau[2] + kc * dT) * area;
                out[3] = tau[2] * area;
            }
            Fv[f] = make_float4(out[0], out[1], out[2], out[3]);
        }
        __syncthreads();
    };
    // the balance of one axis into acc: each thread its own cells (the same ones in every call and in the epilogue), so it
    // shares a phase with the next axis's gradients (disjoint arrays) and needs no barrier before the epilogue
    auto balance = [&](auto axis_c) {
        constexpr int d = decltype(axis_c)::value;
        constexpr int Fd[3] = {TX + (d == 0), TY + (d == 1), TZ + (d == 2)};
        for (int c = tid; c < NC; c += NT) {
            const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
            const int fl = (c3[2] * Fd[1] + c3[1]) * Fd[0] + c3[0];
            const int fr = fl + (d == 0 ? 1 : (d == 1 ? Fd[0] : Fd[0] * Fd[1]));
            const float4 l = Fv[fl], r = Fv[fr];
            const float4 dif = make_float4(r.x - l.x, r.y - l.y, r.z - l.z, r.w - l.w);
            if (d == 0) {
                acc[c] = dif;
            } else {
                const float4 s = acc[c];
                acc[c] = make_float4(s.x + dif.x, s.y + dif.y, s.z + dif.z, s.w + dif.w);
            }
        }
    };
    sweep(std::integral_constant<int, 0>{});
    balance(std::integral_constant<int, 0>{});
    sweep(std::integral_constant<int, 1>{});
    balance(std::integral_constant<int, 1>{});
    sweep(std::integral_constant<int, 2>{});
    balance(std::integral_constant<int, 2>{});
    double smax = 0.0;
    const float gm1 = (float)(a.eos.gamma - 1.0);
    for (int c = tid; c < NC; c += NT) {
        const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
        const int g3[3] = {o3[0] + c3[0], o3[1] + c3[1], o3[2] + c3[2]};
        if (g3[0] >= m.nx || g3[1] >= m.ny || g3[2] >= m.nz) continue;
        const long long cell = ((long long)g3[2] * m.ny + g3[1]) * m.nx + g3[0];
        const float4 s4 = acc[c];
        a.Rvf[cell] = s4.x;
        a.Rvf[m.plane + cell] = s4.y;
        a.Rvf[2 * m.plane + cell] = s4.z;
        a.Rvf[3 * m.plane + cell] = s4.w;
        const int p = bidx(c3[0], c3[1], c3[2]);
        const float rho = vmax(R[p], Num<float>::eos_eps);
        const float4 v = V[p];
        const float T = v.w;
        const float nu_eff = vmax((4.0f / 3.0f) * (mu / rho), (kc * gm1) / rho) + 1e-12f;
        const float vm = vmax(vmax(fabsf(v.x), fabsf(v.y)), fabsf(v.z));
        const float cs = sqrtf((float)a.eos.gamma * (T + (float)a.eos.p_inf / rho));
        const double s = (double)(vm + cs + 2.0f * (float)a.L * (float)a.inv_h2 * nu_eff);
        if (s > smax) smax = s;
    }
    const double bm = block_max<NT>(smax, red);
    if (tid == 0) a.blockmax[b] = bm;
}

// The per-axis sweep's shared memory with TMA boxes (mixed_axis with TMA): red [32 doubles] | the barrier | P | acc | Sf |
// (128-byte aligned) WL, WR, sized for the largest box (16 x 8 x 8 x 5 doubles, 40 KB), which the copy fills while the
// face-value arrays are idle.
template <int TX, int TY, int TZ> struct MixedTmaShape {
    using S = MixedShape<3, kWeno5, TX, TY, TZ>;
    static constexpr int P_OFF = 272, ACC_OFF = P_OFF + 4 * S::NV * S::EXT, SF_OFF = ACC_OFF + 4 * S::NV * S::NC;
    static constexpr int STG_OFF = (SF_OFF + S::FLAG_BYTES + 127) / 128 * 128;
    static constexpr int BOX_BYTES = 16 * TY * TZ * S::NV * 8;   // the x sweep's box, the largest
    static constexpr int STG_BYTES = BOX_BYTES > 8 * S::NV * S::NF ? BOX_BYTES : 8 * S::NV * S::NF;
    static constexpr size_t SMEM_BYTES = STG_OFF + STG_BYTES;
};

// The mixed WENO5-Z stage kernel of a 3-D mesh without part interfaces, non-reflecting sides or an immersed body, whose
// boxes come in by TMA (tma.cuh; no copy multicasts), in two forms chosen per tile (a branch uniform over the CTA):
// - the per-axis sweep of mixed_stage_kernel (mixed_axis with TMA: a 16 x 8 x 8, 8 x 14 x 8 or 8 x 8 x 14 box per axis),
//   for every tile of the ungated kernel and for the gated tiles that keep WENO5-Z along some axis or beside a seam;
// - the cross (gated tiles linear along all three axes and at all six seams): one image of the tile and its three halos
//   (the 8x8x8 tile and 3 cells beyond each of its six faces, 1664 cells) converted once, from a 16 x 8 x 8 box (the tile
//   and its x halos) and four 3-deep halo boxes; then every face of the three axes in one pass, one thread per face and
//   all five variables (the linear face values straight into the Riemann solver, no face-value arrays); then the
//   balance ((0 - x) - y) - z of each cell from the three flux arrays in the epilogue.
// Both forms give the bits of mixed_stage_kernel (the explicitly rounded lin5 / weno5z, balance and update), so a face
// between tiles of the two forms gets one flux. A tile whose boxes would leave the mesh (wrapped or ghost cells) takes the
// index-mapping loader for those parts. Measured at 256^3 (Taylor-Green, every tile-axis linear, with the viscous sums
// and U0): 1.60 ms per launch for the cross against 2.11 ms for the per-axis sweep; with WENO5-Z along every axis the
// per-axis sweep is the faster (2.74 against 3.01 ms for a cross that solved WENO5-Z faces too: the per-axis sweep's
// (face, variable) items spread the WENO5-Z work finer).
// Shared memory: the larger of the two layouts (74.1 KB), three CTAs of 384 threads per SM (at most 56 registers).
struct CrossShape {
    // slots of the cross: the tile's 512 cells in rows of 9 (576 slots: x + 9 y + 72 z, so that a warp reading one x
    // column of 32 rows touches 32 banks), then the six 3-deep halos of 192 cells
    static constexpr int NV = 5, NCORE = 576, NHALO = 192, NPC = NCORE + 6 * NHALO;
    static constexpr int NFA = 576, NFACE = 3 * NFA, NINNER = 448;                    // faces per axis; t = 1 .. 7
    static constexpr int BAR_OFF = 256, P_OFF = 272;
    static constexpr int STG_OFF = (P_OFF + 4 * NV * NPC + 127) / 128 * 128;
    static constexpr int XBOX = 16 * 8 * 8, HBOX = 8 * 3 * 8;   // cells of the x box and of one halo box
    static constexpr int STG_BYTES = XBOX * NV * 8;
    static constexpr size_t CROSS_BYTES = STG_OFF + STG_BYTES;
    static constexpr size_t SMEM_BYTES = CROSS_BYTES > MixedTmaShape<8, 8, 8>::SMEM_BYTES ? CROSS_BYTES : MixedTmaShape<8, 8, 8>::SMEM_BYTES;
    static_assert(4 * HBOX * NV * 8 <= STG_BYTES && 3 * NV * NFA * 4 <= STG_BYTES, "the staging area holds the halo boxes and the fluxes");
};

// the cross's slot of the cell at s along axis A (s in [-3, 11)) and (u, v) along the other two axes in increasing
// order: the tile's cells (x + 9 y + 72 z), then the six halos (axis-major, low side first), each 3 deep x 64 cells
template <int A> __device__ __forceinline__ int cross_slot(int s, int u, int v) {
    if (s < 0) return 576 + (2 * A) * 192 + (s + 3) + 3 * (u + 8 * v);
    if (s >= 8) return 576 + (2 * A + 1) * 192 + (s - 8) + 3 * (u + 8 * v);
    return A == 0 ? s + 9 * u + 72 * v : (A == 1 ? u + 9 * s + 72 * v : u + 9 * v + 72 * s);
}
// cell e of the cross (the tile's 512 cells, x fastest, then the six halos of cross_slot's order): its tile-local
// coordinates and its slot
__device__ __forceinline__ int cross_cell(int e, int l3[3]) {
    if (e < 512) {
        l3[0] = e & 7;
        l3[1] = (e >> 3) & 7;
        l3[2] = e >> 6;
        return l3[0] + 9 * l3[1] + 72 * l3[2];
    }
    const int k = (e - 512) / 192, r = (e - 512) % 192, A = k >> 1;
    const int l = r % 3, uv = r / 3, u = uv & 7, v = uv >> 3;
    const int s = (k & 1) ? 8 + l : l - 3;
    l3[0] = A == 0 ? s : u;
    l3[1] = A == 0 ? u : (A == 1 ? s : v);
    l3[2] = A == 2 ? s : v;
    return e + 64;
}

// One face of axis A in the cross (linear face values): item r of the axis (the 448 faces inside the tile, t = 1 .. 7,
// then the two seam layers t = 0 and 8); its flux goes to Fs at the face's index in mixed_axis's numbering.
template <int A, int RIEMANN>
__device__ __forceinline__ void cross_face(const StageArgs& a, const Eos<float>& ef, float sb, const float* __restrict__ P, float* __restrict__ Fs,
                                           int r, const int o3[3], float& smax) {
    constexpr int NV = 5, NPC = CrossShape::NPC;
    int t, u, v;
    if (r < CrossShape::NINNER) {   // (the lanes of a warp run along the cross's rows: no two on one bank)
        if (A == 0) {
            t = 1 + r % 7;
            u = (r / 7) & 7;
            v = r / 56;
        } else if (A == 1) {
            u = r & 7;
            t = 1 + (r >> 3) % 7;
            v = (r >> 3) / 7;
        } else {
            u = r & 7;
            v = (r >> 3) & 7;
            t = 1 + (r >> 6);
        }
    } else {
        const int q = r - CrossShape::NINNER;
        u = q & 7;
        v = (q >> 3) & 7;
        t = (q >> 6) * 8;
    }
    const int f = A == 0 ? t + 9 * (u + 8 * v) : (A == 1 ? u + 8 * (t + 9 * v) : u + 8 * (v + 8 * t));
    int sl[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) sl[k] = cross_slot<A>(t - 3 + k, u, v);
    St<float, NV> wl, wr;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        const float* c = P + q * NPC;
        const float c0 = c[sl[0]], c1 = c[sl[1]], c2 = c[sl[2]], c3 = c[sl[3]], c4 = c[sl[4]], c5 = c[sl[5]];
        wl[q] = lin5(c0, c1, c2, c3, c4);
        wr[q] = lin5(c5, c4, c3, c2, c1);
    }
    const Mesh& m = a.m;
    const int n3[3] = {m.nx, m.ny, m.nz};
    const int g3[3] = {o3[0] + (A == 0 ? t : u), o3[1] + (A == 0 ? u : (A == 1 ? t : v)), o3[2] + (A == 2 ? t : v)};
    bool inside = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) inside = inside && (d == A ? g3[d] <= n3[d] : g3[d] < n3[d]);
    St<float, NV> F;
#pragma unroll
    for (int q = 0; q < NV; ++q) F[q] = 0.0f;
    // (no face of a tile in the cross form lies on a side without a halo: the gate keeps every tile whose extension along
    // an axis leaves the mesh across a side that is not periodic WENO5-Z along that axis, so such a tile never takes the
    // cross form; mixed_axis's first-order side states are not needed here)
    if (inside) {
        const float sp = face_flux_prim<RIEMANN>(ef, sb, wl, wr, A, F);
        if (sp > smax) smax = sp;
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) Fs[(A * NV + q) * CrossShape::NFA + f] = F[q];
}

// The epilogue's operands that no box brings in (the 8x8x8 tile's rows of U0 and of the FP32 viscous sums) head for L2
// at the start of the tile, so that the epilogue's loads find them there (measured at 256^3 in the cross form: 1.79 ->
// 1.72 ms per launch)
template <int NT> __device__ __forceinline__ void prefetch_epilogue(const StageArgs& a, const int o3[3]) {
    if (a.mode != kCombine && !a.Rvf) return;
    const Mesh& m = a.m;
    for (int k = threadIdx.x; k < 9 * 64; k += NT) {
        const int q = k >> 6, y = o3[1] + (k & 7), z = o3[2] + ((k >> 3) & 7);
        if (y >= m.ny || z >= m.nz) continue;
        const long long row = ((long long)z * m.ny + y) * m.nx + o3[0];
        if (q < 5 && a.mode == kCombine) prefetch_l2(a.U0 + q * m.plane + row);
        if (q >= 5 && a.Rvf) prefetch_l2(a.Rvf + (q - 5) * m.plane + row);
    }
}

// The cross form of a tile (see mixed_stage_kernel_tma): maps m[0] (the 16 x 8 x 8 box), m[3] and m[4] (the y and z halo
// boxes); `phase` counts the barrier's completed copies.
template <int RIEMANN, int NT>
__device__ __forceinline__ void cross_tile(const StageArgs& a, const TmaMaps& maps, unsigned char* smem_b, const int o3[3], unsigned& phase, float& smax) {
    using L = CrossShape;
    constexpr int NV = 5, NPC = L::NPC;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_b + L::BAR_OFF);
    float* P = reinterpret_cast<float*>(smem_b + L::P_OFF);
    double* stg = reinterpret_cast<double*>(smem_b + L::STG_OFF);
    float* Fs = reinterpret_cast<float*>(smem_b + L::STG_OFF);
    const Mesh& m = a.m;
    const int n3[3] = {m.nx, m.ny, m.nz};
    const Eos<float> ef{a.eos.type, (float)a.eos.gamma, (float)a.eos.p_inf};
    const float sb = (float)a.shock_blend;
    const int tid = threadIdx.x;
    const bool aligned = (tma::su32(stg) & 127u) == 0;
    // every thread waits for the barrier's current phase, at most 2^22 polls; a copy that never completes stops the run
    // (status 5) instead of hanging the GPU
    auto wait = [&]() -> bool {
        bool done = false;
        for (int it = 0; it < (1 << 22) && !done; ++it) done = tma::mbar_try_wait(bar, phase & 1u);
        ++phase;
        if (!done && tid == 0) atomicExch(const_cast<int*>(&a.ctl->status), 5);
        return done;
    };
    // cells e0 .. e1 of the cross by index mapping (wrapped and ghost cells), the primitive state recovered in FP64
    auto load_slots = [&](int e0, int e1) {
        for (int e = e0 + tid; e < e1; e += NT) {
            int l3[3];
            const int p = cross_cell(e, l3);
            const St<double, NV> w = c2p(a.eos, stencil_cons<3, NV, false>(m, a.bc, a.eos, a.U, o3[0] + l3[0], o3[1] + l3[1], o3[2] + l3[2]));
#pragma unroll
            for (int q = 0; q < NV; ++q) P[q * NPC + p] = (float)w[q];
        }
    };
    prefetch_epilogue<NT>(a, o3);
    // ---- 1. the tile and its x halos (cells 0 .. 895): one 16 x 8 x 8 box from x = o - 4
    if (aligned && o3[0] >= 4 && o3[0] + 12 <= n3[0] && o3[1] + 8 <= n3[1] && o3[2] + 8 <= n3[2]) {
        if (tid == 0) {
            tma::fence_proxy_async();
            tma::mbar_expect_tx(bar, (unsigned)(L::XBOX * NV * 8));
            tma::load_4d(stg, &maps.m[0], o3[0] - 4, o3[1], o3[2], 0, bar);
        }
        const bool done = wait();
        for (int e = tid; e < 14 * 64; e += NT) {
            const int xl = e % 14 - 3, y = (e / 14) & 7, z = e / 112;
            const int si = (z * 8 + y) * 16 + xl + 4;
            St<double, NV> uc;
#pragma unroll
            for (int q = 0; q < NV; ++q) uc[q] = done ? stg[q * L::XBOX + si] : 1.0;
            const St<double, NV> w = c2p(a.eos, uc);
            const int p = cross_slot<0>(xl, y, z);
#pragma unroll
            for (int q = 0; q < NV; ++q) P[q * NPC + p] = (float)w[q];
        }
    } else {
        load_slots(0, 896);
    }
    __syncthreads();
    // ---- 2. the y and z halos (cells 896 .. 1663): four 3-deep boxes on one barrier phase
    if (aligned && o3[1] >= 3 && o3[1] + 11 <= n3[1] && o3[2] >= 3 && o3[2] + 11 <= n3[2] && o3[0] + 8 <= n3[0]) {
        if (tid == 0) {
            tma::fence_proxy_async();
            tma::mbar_expect_tx(bar, (unsigned)(4 * L::HBOX * NV * 8));
            tma::load_4d(stg, &maps.m[3], o3[0], o3[1] - 3, o3[2], 0, bar);
            tma::load_4d(stg + 1 * L::HBOX * NV, &maps.m[3], o3[0], o3[1] + 8, o3[2], 0, bar);
            tma::load_4d(stg + 2 * L::HBOX * NV, &maps.m[4], o3[0], o3[1], o3[2] - 3, 0, bar);
            tma::load_4d(stg + 3 * L::HBOX * NV, &maps.m[4], o3[0], o3[1], o3[2] + 8, 0, bar);
        }
        const bool done = wait();
        for (int e = tid; e < 4 * L::HBOX; e += NT) {
            const int k = e / L::HBOX, r = e % L::HBOX;
            const double* box = stg + k * L::HBOX * NV;
            int si, p;
            if (k < 2) {   // 8 x 3 x 8 boxes below and above the tile along y
                const int x = r & 7, yb = (r >> 3) % 3, z = r / 24;
                si = (z * 3 + yb) * 8 + x;
                p = cross_slot<1>(k == 0 ? yb - 3 : 8 + yb, x, z);
            } else {       // 8 x 8 x 3 boxes along z
                const int x = r & 7, y = (r >> 3) & 7, zb = r >> 6;
                si = (zb * 8 + y) * 8 + x;
                p = cross_slot<2>(k == 2 ? zb - 3 : 8 + zb, x, y);
            }
            St<double, NV> uc;
#pragma unroll
            for (int q = 0; q < NV; ++q) uc[q] = done ? box[q * L::HBOX + si] : 1.0;
            const St<double, NV> w = c2p(a.eos, uc);
#pragma unroll
            for (int q = 0; q < NV; ++q) P[q * NPC + p] = (float)w[q];
        }
    } else {
        load_slots(896, 1664);
    }
    __syncthreads();
    // ---- 3. every face of the three axes (the faces inside the tile first, 448 per axis, then the seam layers)
    for (int it = tid; it < L::NFACE; it += NT) {
        int A, r;
        if (it < 3 * L::NINNER) {
            A = it / L::NINNER;
            r = it - A * L::NINNER;
        } else {
            const int q = it - 3 * L::NINNER;
            A = q >> 7;
            r = L::NINNER + (q & 127);
        }
        if (A == 0)
            cross_face<0, RIEMANN>(a, ef, sb, P, Fs, r, o3, smax);
        else if (A == 1)
            cross_face<1, RIEMANN>(a, ef, sb, P, Fs, r, o3, smax);
        else
            cross_face<2, RIEMANN>(a, ef, sb, P, Fs, r, o3, smax);
    }
    __syncthreads();
    // ---- 4. the balance ((0 - x) - y) - z, the residual widened to FP64 and the FP64 stage update
    const float Ax = (float)m.area[0], Ay = (float)m.area[1], Az = (float)m.area[2];
    const double dt = a.ctl->dt;
    for (int c = tid; c < 512; c += NT) {
        const int c3[3] = {c & 7, (c >> 3) & 7, c >> 6};
        const int g3[3] = {o3[0] + c3[0], o3[1] + c3[1], o3[2] + c3[2]};
        if (g3[0] >= m.nx || g3[1] >= m.ny || g3[2] >= m.nz) continue;
        const long long cell = ((long long)g3[2] * m.ny + g3[1]) * m.nx + g3[0];
        const int fx = (c3[2] * 8 + c3[1]) * 9 + c3[0], fy = (c3[2] * 9 + c3[1]) * 8 + c3[0], fz = c;
        CellIn<NV> in;
        cell_load(a, cell, in);
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const float* X = Fs + (0 * NV + q) * L::NFA;
            const float* Y = Fs + (1 * NV + q) * L::NFA;
            const float* Z = Fs + (2 * NV + q) * L::NFA;
            float acc = -__fmul_rn(X[fx + 1] - X[fx], Ax);
            acc = __fmaf_rn(-(Y[fy + 8] - Y[fy]), Ay, acc);
            acc = __fmaf_rn(-(Z[fz + 64] - Z[fz]), Az, acc);
            a.out[q * m.plane + cell] = cell_out(a, in, q, acc, dt);
        }
    }
}

// whether a gated tile is linear along all three axes and at all six seams (the seam rule of mixed_axis)
__device__ __forceinline__ bool tile_all_linear(const StageArgs& a, int b, const int o3[3]) {
    const long long nt3 = (long long)a.tiles[0] * a.tiles[1] * a.tiles[2];
    bool lin = true;
#pragma unroll
    for (int A = 0; A < 3; ++A) {
        const unsigned char* fl = a.sens_flags + A * nt3;
        const int nt = a.tiles[A];
        const int st = A == 0 ? 1 : (A == 1 ? a.tiles[0] : a.tiles[0] * a.tiles[1]);
        const int ta = A == 0 ? b % a.tiles[0] : (A == 1 ? (b / a.tiles[0]) % a.tiles[1] : b / (a.tiles[0] * a.tiles[1]));
        const bool wrap_lo = a.bc.halo[2 * A] == kHaloWrap, wrap_hi = a.bc.halo[2 * A + 1] == kHaloWrap;
        lin = lin && fl[b] == 0;
        lin = lin && (ta > 0 ? fl[b - st] == 0 : (wrap_lo ? fl[b + (nt - 1) * st] == 0 : true));
        lin = lin && (ta < nt - 1 ? fl[b + st] == 0 : (wrap_hi ? fl[b - (nt - 1) * st] == 0 : true));
    }
    return lin;
}

template <int RIEMANN, int NT, bool GATED>
__global__ void __launch_bounds__(NT, 3) mixed_stage_kernel_tma(const StageArgs a, const __grid_constant__ TmaMaps maps) {
    using S = MixedShape<3, kWeno5, 8, 8, 8>;
    using LO = MixedTmaShape<8, 8, 8>;
    constexpr int NV = S::NV, NC = S::NC;
    extern __shared__ __align__(128) unsigned char smem_b[];
    double* red = reinterpret_cast<double*>(smem_b);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_b + CrossShape::BAR_OFF);
    if (!*a.gate) return;
    if (threadIdx.x == 0) {
        tma::mbar_init(bar, 1);
        tma::fence_mbar_init();
    }
    __syncthreads();
    const Mesh& m = a.m;
    const int tid = threadIdx.x, b = blockIdx.x + a.b0;
    const int o3[3] = {(b % a.tiles[0]) * 8, ((b / a.tiles[0]) % a.tiles[1]) * 8, (b / (a.tiles[0] * a.tiles[1])) * 8};
    float smax = 0.0f;
    unsigned phase = 0;
    bool cross = false;
    if constexpr (GATED) cross = tile_all_linear(a, b, o3);
    if (cross) {
        cross_tile<RIEMANN, NT>(a, maps, smem_b, o3, phase, smax);
    } else {
        prefetch_epilogue<NT>(a, o3);
        float* P = reinterpret_cast<float*>(smem_b + LO::P_OFF);
        float* acc = reinterpret_cast<float*>(smem_b + LO::ACC_OFF);
        unsigned char* Sf = smem_b + LO::SF_OFF;
        float* WL = reinterpret_cast<float*>(smem_b + LO::STG_OFF);
        float* WR = WL + NV * S::NF;
        const Eos<float> ef{a.eos.type, (float)a.eos.gamma, (float)a.eos.p_inf};
        const float sb = (float)a.shock_blend, weps = (float)a.weno_eps;
        mixed_axis<0, 3, kWeno5, RIEMANN, 8, 8, 8, NT, GATED, false, true>(a, ef, sb, weps, P, WL, WR, acc, Sf, o3, smax, maps.m, bar, &phase);
        mixed_axis<1, 3, kWeno5, RIEMANN, 8, 8, 8, NT, GATED, false, true>(a, ef, sb, weps, P, WL, WR, acc, Sf, o3, smax, maps.m, bar, &phase);
        mixed_axis<2, 3, kWeno5, RIEMANN, 8, 8, 8, NT, GATED, false, true>(a, ef, sb, weps, P, WL, WR, acc, Sf, o3, smax, maps.m, bar, &phase);
        const double dt = a.ctl->dt;
        for (int c = tid; c < NC; c += NT) {
            const int c3[3] = {c % 8, (c / 8) % 8, c / 64};
            const int g3[3] = {o3[0] + c3[0], o3[1] + c3[1], o3[2] + c3[2]};
            if (g3[0] >= m.nx || g3[1] >= m.ny || g3[2] >= m.nz) continue;
            const long long cell = ((long long)g3[2] * m.ny + g3[1]) * m.nx + g3[0];
            CellIn<NV> in;
            cell_load(a, cell, in);
#pragma unroll
            for (int q = 0; q < NV; ++q) a.out[q * m.plane + cell] = cell_out(a, in, q, acc[q * NC + c], dt);
        }
    }
    const double bm = block_max<NT>((double)smax, red);
    if (tid == 0) a.blockmax[b] = bm;
}

}   // namespace fvg
