// The MUSCL-Hancock residual of a 2-D mesh, fused with its update: the limited face states of every cell, advanced by
// half a step with the cell's own flux difference (predictor), then the Riemann solves and the flux balance
// (MusclReconstruction::hancock_residual_2d, cpp/src/Schemes.cpp:2135-2477 and 2782-2830).
//
// A CTA owns a TX x TY tile:
//   1. the primitive state of the tile and two cells around it (boundary conditions by index mapping);
//   2. the four limited states (low / high side along x and y) of the tile's cells and of the ring of cells around it,
//      predicted for every cell of the mesh (the ring's wrapped cells of a periodic axis included); a ring position
//      beyond another side keeps the unpredicted state, which is what the reference puts on a face of a side with a
//      ghost slab (stencil_face_state); at a side without a halo the cell's own state there is the round trip of the
//      cell (hancock_row); a state the predictor would make inadmissible stays as it was (hancock_cell);
//   3. the x faces, then the y faces: left state = high-side state of the cell before the face, right state = low-side
//      state of the cell after it; on a wall side the ghost is the wall state of the predicted cell state, on a side
//      without a halo the round trip of the first-order ghost (hancock_xfaces / hancock_yfaces);
//   4. the balance ((0 - (Fr dy - Fl dy)) - (Ft dx - Fb dx)) / area and the update U + dt R (or R alone).
#pragma once

#include <type_traits>

#include "grid.cuh"

namespace fvg {

struct HancockArgs {
    Mesh m;
    Bc bc;
    Eos<double> eos;
    double shock_blend;
    int limiter;
    int mode;          // kStoreR or kAxpy
    const double* U;
    const double* Rv;  // the viscous residual of U (null: inviscid); it joins the balance, not the predictor
    double* out;
    double* blockmax;
    const Ctl* ctl;    // dt and half_dt
    const int* gate;
    int tiles[3];
};

template <int TX, int TY> struct HancockShape {
    static constexpr int PX = TX + 4, PY = TY + 4;   // primitive box
    static constexpr int BX = TX + 2, BY = TY + 2;   // predicted-state box
    static constexpr int NF = (TX + 1) * TY > TX * (TY + 1) ? (TX + 1) * TY : TX * (TY + 1);
    // P [4][PX*PY], S [4 states][4][BX*BY], F [4][NF], acc [4][TX*TY], red [32]
    static constexpr int SMEM_DOUBLES = 4 * PX * PY + 16 * BX * BY + 4 * NF + 4 * TX * TY + 32;
    static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;
};

// euler_flux_axis (Schemes.cpp:2137-2141) of a planar state
__device__ __forceinline__ St<double, 4> euler_flux2(const Eos<double>& e, const St<double, 4>& U, int a) {
    const St<double, 4> W = c2p(e, U);
    const double un = a == 0 ? W[1] : W[2], p = W[3];
    St<double, 4> F;
    F[0] = U[0] * un;
    F[1] = U[1] * un + (a == 0 ? p : 0.0);
    F[2] = U[2] * un + (a == 1 ? p : 0.0);
    F[3] = (U[3] + p) * un;
    return F;
}

// admissible_state (Schemes.cpp:2145-2148): rho > floor and p + p_inf > 0, NaN inadmissible
__device__ __forceinline__ bool admissible(const Eos<double>& e, const St<double, 4>& U) {
    if (!(U[0] > Num<double>::eos_eps)) return false;
    return 0.5 * (U[1] * U[1] + U[2] * U[2] + 0.0 * 0.0) < U[0] * (U[3] - e.p_inf);
}

// The source field of a MUSCL-Hancock residual (Simulation::assemble, cpp/src/Simulation.cpp:975-980): zero, then the
// body force and the case's source terms added (RhsSourceTerms::apply_uniform); the predictor takes d - half_dt src, the
// balance R + src after the viscous term (:1043-1047).
template <int NV> __device__ __forceinline__ St<double, NV> body_source(const Bc& bc, const double* U, long long plane, long long cell) {
    St<double, NV> src;
#pragma unroll
    for (int q = 0; q < NV; ++q) src[q] = 0.0;
    if (bc.grav_on) add_body_force<NV>(bc, read_state<NV>(bc, U, plane, cell), src);
    if (bc.src) add_source<NV>(bc, plane, cell, src);
    return src;
}

// FULL = false: a run without part interfaces, non-reflecting sides or the body force (their code compiled out)
template <int RIEMANN, int TX, int TY, int NT, bool FULL = true>
__global__ void __launch_bounds__(NT) hancock_kernel(const HancockArgs a) {
    using S = HancockShape<TX, TY>;
    constexpr int PX = S::PX, PY = S::PY, BX = S::BX, BY = S::BY, NB = BX * BY, NP = PX * PY, NC = TX * TY;
    extern __shared__ double smem[];
    double* P = smem;                  // [4][NP]
    double* Sx = P + 4 * NP;           // [state 0..3: xl, xr, yb, yt][4][NB]
    double* Fl = Sx + 16 * NB;         // [4][NF]
    double* acc = Fl + 4 * S::NF;      // [4][NC]
    double* red = acc + 4 * NC;
    if (!*a.gate) return;
    const Mesh& m = a.m;
    const Eos<double>& e = a.eos;
    const int tid = threadIdx.x, b = blockIdx.x;
    const int ox = (b % a.tiles[0]) * TX, oy = (b / a.tiles[0]) * TY;
    const int nx = m.nx, ny = m.ny;
    const double half_dt = a.ctl->half_dt;
    const double hx = half_dt / m.dx, hy = half_dt / m.dy;

    // ---- 1. primitive box: cells ox-2 .. ox+TX+1, oy-2 .. oy+TY+1
    for (int p = tid; p < NP; p += NT) {
        const int i = ox + p % PX - 2, j = oy + p / PX - 2;
        const St<double, 4> w = c2p(e, stencil_cons<2, 4, FULL>(m, a.bc, e, a.U, i, j, 0));
#pragma unroll
        for (int q = 0; q < 4; ++q) P[q * NP + p] = w[q];
    }
    __syncthreads();
    // ---- 2. the four states of the cells ox-1 .. ox+TX, oy-1 .. oy+TY (not the four corners)
    const bool wrap_x = a.bc.halo[0] == kHaloWrap, wrap_y = a.bc.halo[2] == kHaloWrap;
    for (int p = tid; p < NB; p += NT) {
        const int bi = p % BX, bj = p / BX;
        if ((bi == 0 || bi == BX - 1) && (bj == 0 || bj == BY - 1)) continue;
        const int gi = ox + bi - 1, gj = oy + bj - 1;
        const int pc = (bj + 1) * PX + (bi + 1);   // the cell in the primitive box
        St<double, 4> st[4];
        // muscl_cell_states_line (Schemes.cpp:2204-2229): hi = c + 1/2 phi(c - cm, cp - c), lo = c - 1/2 phi(cp - c, c - cm)
#pragma unroll
        for (int ax = 0; ax < 2; ++ax) {
            const int s = ax == 0 ? 1 : PX;
            St<double, 4> wl, wr;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double cm = P[q * NP + pc - s], c = P[q * NP + pc], cp = P[q * NP + pc + s];
                wl[q] = c + 0.5 * limiter(a.limiter, c - cm, cp - c);
                wr[q] = c - 0.5 * limiter(a.limiter, cp - c, c - cm);
            }
            st[2 * ax + 1] = p2c(e, wl);
            st[2 * ax] = p2c(e, wr);
        }
        // a real cell: of the mesh, of a periodic wrap, or of the neighbouring part beyond a part interface
        const bool real = gi >= -1 && gi <= nx && gj >= -1 && gj <= ny && (wrap_x || held<FULL>(a.bc, 0, gi, nx)) && (wrap_y || held<FULL>(a.bc, 1, gj, ny));
        if (real) {
            // the mesh cell (wrapped): sides without a halo give it the round trip of its own state there
            const int ci = wrap_x ? (gi + nx) % nx : gi, cj = wrap_y ? (gj + ny) % ny : gj;
            const bool b0 = ci == 0 && a.bc.halo[0] == kHaloNone, b1 = ci == nx - 1 && a.bc.halo[1] == kHaloNone;
            const bool b2 = cj == 0 && a.bc.halo[2] == kHaloNone, b3 = cj == ny - 1 && a.bc.halo[3] == kHaloNone;
            if (b0 || b1 || b2 || b3) {
                const St<double, 4> rt = round_trip(e, read_state<4>(a.bc, a.U, m.plane, (long long)cj * nx + ci));
                if (b0) st[0] = rt;
                if (b1) st[1] = rt;
                if (b2) st[2] = rt;
                if (b3) st[3] = rt;
            }
            // an immersed body: its cells are not predicted, nor the sides of a cell that face one (the states of those
            // sides keep the time level of the ghost cells; solid_side_mask, Schemes.cpp:2890-2905, no wrap-around)
            const unsigned char* sol = a.bc.solid;
            const bool is_solid = sol && sol[(long long)cj * nx + ci];
            int sd = 0;
            if (sol && !is_solid) {
                sd = (ci > 0 && sol[(long long)cj * nx + ci - 1] ? 1 : 0) | (ci < nx - 1 && sol[(long long)cj * nx + ci + 1] ? 2 : 0) |
                     (cj > 0 && sol[(long long)(cj - 1) * nx + ci] ? 4 : 0) | (cj < ny - 1 && sol[(long long)(cj + 1) * nx + ci] ? 8 : 0);
            }
            if (!is_solid) {
                // hancock_cell (Schemes.cpp:2153-2172)
                const St<double, 4> fxl = euler_flux2(e, st[0], 0), fxr = euler_flux2(e, st[1], 0);
                const St<double, 4> fyb = euler_flux2(e, st[2], 1), fyt = euler_flux2(e, st[3], 1);
                St<double, 4> d;
#pragma unroll
                for (int q = 0; q < 4; ++q) d[q] = hx * (fxr[q] - fxl[q]) + hy * (fyt[q] - fyb[q]);
                if (FULL && (a.bc.grav_on || a.bc.src)) {   // the body force and the sources join the predictor: d - half_dt src
                    const St<double, 4> src = body_source<4>(a.bc, a.U, m.plane, (long long)cj * nx + ci);
#pragma unroll
                    for (int q = 0; q < 4; ++q) d[q] = d[q] - half_dt * src[q];
                }
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    if (sd & (1 << s)) continue;
                    St<double, 4> n;
#pragma unroll
                    for (int q = 0; q < 4; ++q) n[q] = st[s][q] - d[q];
                    if (admissible(e, n)) st[s] = n;
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int q = 0; q < 4; ++q) Sx[(s * 4 + q) * NB + p] = st[s][q];
    }
    __syncthreads();
    double smax = 0.0;
    // ---- 3. faces: axis 0 (x), then axis 1 (y)
#pragma unroll 1
    for (int axis = 0; axis < 2; ++axis) {
        const int FX = TX + (axis == 0), FY = TY + (axis == 1);
        const int nF = FX * FY;
        const int lo_side = 2 * axis, hi_side = lo_side + 1;
        const bool wall_lo = a.bc.type[lo_side] == kBcWall || a.bc.type[lo_side] == kBcNoSlip || a.bc.type[lo_side] == kBcMovingWall;
        const bool wall_hi = a.bc.type[hi_side] == kBcWall || a.bc.type[hi_side] == kBcNoSlip || a.bc.type[hi_side] == kBcMovingWall;
        for (int f = tid; f < nF; f += NT) {
            const int fi = f % FX, fj = f / FX;
            const int gi = ox + fi, gj = oy + fj;
            const int n_a = axis == 0 ? nx : ny, t = axis == 0 ? gi : gj;
            const bool inside = axis == 0 ? (gi <= nx && gj < ny) : (gi < nx && gj <= ny);
            St<double, 4> F;
#pragma unroll
            for (int q = 0; q < 4; ++q) F[q] = 0.0;
            if (inside) {
                // the cells before and after the face in the state box
                const int pR = (fj + 1) * BX + (fi + 1);
                const int pL = axis == 0 ? pR - 1 : pR - BX;
                const int sL = axis == 0 ? 1 : 3, sR = axis == 0 ? 0 : 2;   // high-side state of L, low-side state of R
                St<double, 4> UL, UR;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    UL[q] = Sx[(sL * 4 + q) * NB + pL];
                    UR[q] = Sx[(sR * 4 + q) * NB + pR];
                }
                if (t == 0) {
                    if (wall_lo)
                        UL = ghost_state(e, a.bc, lo_side, UR);
                    else if (a.bc.halo[lo_side] == kHaloNone)
                        UL = round_trip(e, side_ghost<4, FULL>(m, a.bc, e, a.U, lo_side, gi, gj, 0));
                }
                if (t == n_a) {
                    const int ci = axis == 0 ? nx - 1 : gi, cj = axis == 0 ? gj : ny - 1;
                    if (wall_hi)
                        UR = ghost_state(e, a.bc, hi_side, UL);
                    else if (a.bc.halo[hi_side] == kHaloNone)
                        UR = round_trip(e, side_ghost<4, FULL>(m, a.bc, e, a.U, hi_side, ci, cj, 0));
                }
                const double s = face_flux<RIEMANN>(e, a.shock_blend, UL, UR, axis, F);
                if (s > smax) smax = s;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) Fl[q * S::NF + f] = F[q];
        }
        __syncthreads();
        const double A = m.area[axis];
        for (int c = tid; c < NC; c += NT) {
            const int ci = c % TX, cj = c / TX;
            const int fl = cj * FX + ci, fr = fl + (axis == 0 ? 1 : FX);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double dd = Fl[q * S::NF + fr] * A - Fl[q * S::NF + fl] * A;
                acc[q * NC + c] = axis == 0 ? 0.0 - dd : acc[q * NC + c] - dd;
            }
        }
        __syncthreads();
    }
    // ---- 4. the residual and the update
    const double dt = a.ctl->dt;
    for (int c = tid; c < NC; c += NT) {
        const int gi = ox + c % TX, gj = oy + c / TX;
        if (gi >= nx || gj >= ny) continue;
        const long long cell = (long long)gj * nx + gi;
        St<double, 4> r;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            r[q] = acc[q * NC + c] * m.inv_cell;
            if (a.Rv) r[q] = r[q] + a.Rv[q * m.plane + cell];
        }
        if (FULL && (a.bc.grav_on || a.bc.src)) {
            const St<double, 4> src = body_source<4>(a.bc, a.U, m.plane, cell);
#pragma unroll
            for (int q = 0; q < 4; ++q) r[q] = r[q] + src[q];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const long long x = q * m.plane + cell;
            a.out[x] = a.mode == 0 ? r[q] : a.U[x] + dt * r[q];
        }
    }
    const double bm = block_max<NT>(smax, red);
    if (tid == 0) a.blockmax[b] = bm;
}

}   // namespace fvg

namespace fvg {

// ---------------------------------------------------------------------------------------------- 3-D MUSCL-Hancock
// MusclReconstruction::hancock_residual_3d (cpp/src/Schemes.cpp:2488-2769, 2832-2888) on a TX x TY x TZ tile:
//   1. the primitive state of the tile and two cells around it;
//   2. for the tile and the cells across its faces (the tile +- 1, at most one axis outside), the predictor increment of
//      every real cell (a cell of the mesh, or the wrapped cell of a periodic axis): the six limited states (low / high
//      along x, y, z; at a side without a halo the cell's own round trip), their Euler fluxes and
//      d = (hx (fxr - fxl) + hy (fyt - fyb)) + hz (fzk - fzf) (hancock_cell_3d_impl); not for a solid cell or a position
//      beyond a side that is not periodic (whose state the reference keeps unpredicted, stencil_face_state3);
//   3. per axis, the faces: each recomputes the two limited states it needs and applies the cell's increment (a state
//      that would be inadmissible, or one facing a solid cell, stays), the wall ghost of the predicted state on a wall
//      side, the round trip of the first-order ghost on a side without a halo; Riemann solve; balance
//      ((0 - x) - y) - z (hancock_xfaces3 / yfaces3 / zfaces3 and the balance of hancock_residual_3d_impl);
//   4. R / volume and the update U + dt R (or R alone).
template <int TX, int TY, int TZ> struct Hancock3Shape {
    static constexpr int PX = TX + 4, PY = TY + 4, PZ = TZ + 4, NP = PX * PY * PZ;   // primitive box
    static constexpr int DX = TX + 2, DY = TY + 2, DZ = TZ + 2, ND = DX * DY * DZ;   // increment box
    static constexpr int cmax(int a, int b) { return a > b ? a : b; }
    static constexpr int NF = cmax(cmax((TX + 1) * TY * TZ, TX * (TY + 1) * TZ), TX * TY * (TZ + 1));
    static constexpr int NC = TX * TY * TZ;
    // doubles: P [5][NP], D [5][ND], F [5][NF], acc [5][NC], red [32]; bytes: flags [ND] (bit 6: predicted, bits 0-5: sides
    // facing a solid cell)
    static constexpr int SMEM_DOUBLES = 5 * NP + 5 * ND + 5 * NF + 5 * NC + 32;
    static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES + (ND + 15) / 16 * 16;
};

// euler_flux_axis3 (Schemes.cpp:2176-2180)
__device__ __forceinline__ St<double, 5> euler_flux3(const Eos<double>& e, const St<double, 5>& U, int a) {
    const St<double, 5> W = c2p(e, U);
    const double un = a == 0 ? W[1] : (a == 1 ? W[2] : W[4]), p = W[3];
    St<double, 5> F;
    F[0] = U[0] * un;
    F[1] = U[1] * un + (a == 0 ? p : 0.0);
    F[2] = U[2] * un + (a == 1 ? p : 0.0);
    F[3] = (U[3] + p) * un;
    F[4] = U[4] * un + (a == 2 ? p : 0.0);
    return F;
}

__device__ __forceinline__ bool admissible3(const Eos<double>& e, const St<double, 5>& U) {
    if (!(U[0] > Num<double>::eos_eps)) return false;
    return 0.5 * (U[1] * U[1] + U[2] * U[2] + U[4] * U[4]) < U[0] * (U[3] - e.p_inf);
}

template <int RIEMANN, int TX, int TY, int TZ, int NT, bool FULL = true>
__global__ void __launch_bounds__(NT) hancock3d_kernel(const HancockArgs a) {
    using S = Hancock3Shape<TX, TY, TZ>;
    constexpr int PX = S::PX, PY = S::PY, NP = S::NP, DX = S::DX, DY = S::DY, ND = S::ND, NC = S::NC;
    extern __shared__ double smem[];
    double* P = smem;                  // [5][NP]
    double* D = P + 5 * NP;            // [5][ND]
    double* Fl = D + 5 * ND;           // [5][NF]
    double* acc = Fl + 5 * S::NF;      // [5][NC]
    double* red = acc + 5 * NC;
    unsigned char* flg = reinterpret_cast<unsigned char*>(red + 32);   // [ND]
    if (!*a.gate) return;
    const Mesh& m = a.m;
    const Eos<double>& e = a.eos;
    const int tid = threadIdx.x, b = blockIdx.x;
    const int o3[3] = {(b % a.tiles[0]) * TX, ((b / a.tiles[0]) % a.tiles[1]) * TY, (b / (a.tiles[0] * a.tiles[1])) * TZ};
    const int n3[3] = {m.nx, m.ny, m.nz};
    const double half_dt = a.ctl->half_dt;
    const double hx = half_dt / m.dx, hy = half_dt / m.dy, hz = half_dt / m.dz;
    const bool wrap[3] = {a.bc.halo[0] == kHaloWrap, a.bc.halo[2] == kHaloWrap, a.bc.halo[4] == kHaloWrap};
    auto pidx = [&](int i, int j, int k) { return ((k + 2) * PY + (j + 2)) * PX + (i + 2); };   // tile-relative -2 .. T+1
    auto didx = [&](int i, int j, int k) { return ((k + 1) * DY + (j + 1)) * DX + (i + 1); };   // tile-relative -1 .. T
    auto cell_of = [&](int ci, int cj, int ck) { return ((long long)ck * m.ny + cj) * m.nx + ci; };

    // ---- 1. primitive box
    for (int p = tid; p < NP; p += NT) {
        const int i = o3[0] + p % PX - 2, j = o3[1] + (p / PX) % PY - 2, k = o3[2] + p / (PX * PY) - 2;
        const St<double, 5> w = c2p(e, stencil_cons<3, 5, FULL>(m, a.bc, e, a.U, i, j, k));
#pragma unroll
        for (int q = 0; q < 5; ++q) P[q * NP + p] = w[q];
    }
    __syncthreads();

    // the limited state of side s (0 low x, 1 high x, 2 low y, ...) of the cell at tile-relative (li, lj, lk): MUSCL of the
    // primitive box (hi = c + 1/2 phi(c - cm, cp - c), lo = c - 1/2 phi(cp - c, c - cm)), or the round trip of the cell's
    // own state at a side without a halo (hancock_row3)
    auto limited = [&](int li, int lj, int lk, int s) {
        const int ax = s >> 1;
        const int st = ax == 0 ? 1 : (ax == 1 ? PX : PX * PY);
        const int pc = pidx(li, lj, lk);
        St<double, 5> w;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double cm = P[q * NP + pc - st], c = P[q * NP + pc], cp = P[q * NP + pc + st];
            w[q] = (s & 1) ? c + 0.5 * limiter(a.limiter, c - cm, cp - c) : c - 0.5 * limiter(a.limiter, cp - c, c - cm);
        }
        St<double, 5> u = p2c(e, w);
        const int g[3] = {o3[0] + li, o3[1] + lj, o3[2] + lk};
        int c3[3];
        bool real = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            real = real && g[d] >= -1 && g[d] <= n3[d] && (wrap[d] || held<FULL>(a.bc, d, g[d], n3[d]));
            c3[d] = wrap[d] ? (g[d] + n3[d]) % n3[d] : g[d];
        }
        if (real) {
            const int side_lo = 2 * ax, c = c3[ax];
            const bool at = (s & 1) ? (c == n3[ax] - 1 && a.bc.halo[side_lo + 1] == kHaloNone) : (c == 0 && a.bc.halo[side_lo] == kHaloNone);
            if (at) u = round_trip(e, read_state<5>(a.bc, a.U, m.plane, cell_of(c3[0], c3[1], c3[2])));
        }
        return u;
    };

    // ---- 2. predictor increments of the tile +- 1 (positions outside the tile along at most one axis)
    for (int p = tid; p < ND; p += NT) {
        const int li = p % DX - 1, lj = (p / DX) % DY - 1, lk = p / (DX * DY) - 1;
        const int out = (li < 0 || li >= TX) + (lj < 0 || lj >= TY) + (lk < 0 || lk >= TZ);
        unsigned char f = 0;
        St<double, 5> d;
#pragma unroll
        for (int q = 0; q < 5; ++q) d[q] = 0.0;
        if (out <= 1) {
            const int g[3] = {o3[0] + li, o3[1] + lj, o3[2] + lk};
            bool real = true;
            int c3[3];
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                real = real && g[x] >= -1 && g[x] <= n3[x] && (wrap[x] || held<FULL>(a.bc, x, g[x], n3[x]));
                c3[x] = wrap[x] ? (g[x] + n3[x]) % n3[x] : g[x];
            }
            const unsigned char* sol = a.bc.solid;
            const bool is_solid = real && sol && sol[cell_of(c3[0], c3[1], c3[2])];
            if (real && !is_solid) {
                St<double, 5> st[6];
#pragma unroll
                for (int s = 0; s < 6; ++s) st[s] = limited(li, lj, lk, s);
                const St<double, 5> fxl = euler_flux3(e, st[0], 0), fxr = euler_flux3(e, st[1], 0);
                const St<double, 5> fyb = euler_flux3(e, st[2], 1), fyt = euler_flux3(e, st[3], 1);
                const St<double, 5> fzf = euler_flux3(e, st[4], 2), fzk = euler_flux3(e, st[5], 2);
#pragma unroll
                for (int q = 0; q < 5; ++q) d[q] = (hx * (fxr[q] - fxl[q]) + hy * (fyt[q] - fyb[q])) + hz * (fzk[q] - fzf[q]);
                if (FULL && (a.bc.grav_on || a.bc.src)) {
                    const St<double, 5> src = body_source<5>(a.bc, a.U, m.plane, cell_of(c3[0], c3[1], c3[2]));
#pragma unroll
                    for (int q = 0; q < 5; ++q) d[q] = d[q] - half_dt * src[q];
                }
                f = 64;
                if (sol) {   // solid_side_mask (Schemes.cpp:2890-2905), no wrap-around
                    auto sd = [&](int i, int j, int k) { return i >= 0 && i < n3[0] && j >= 0 && j < n3[1] && k >= 0 && k < n3[2] && sol[cell_of(i, j, k)]; };
                    const int i = c3[0], j = c3[1], k = c3[2];
                    f |= (sd(i - 1, j, k) ? 1 : 0) | (sd(i + 1, j, k) ? 2 : 0) | (sd(i, j - 1, k) ? 4 : 0) | (sd(i, j + 1, k) ? 8 : 0) |
                         (sd(i, j, k - 1) ? 16 : 0) | (sd(i, j, k + 1) ? 32 : 0);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) D[q * ND + p] = d[q];
        flg[p] = f;
    }
    __syncthreads();

    // the predicted state of side s of the cell at tile-relative (li, lj, lk) (hancock_cell_3d_impl for one state)
    auto predicted = [&](int li, int lj, int lk, int s) {
        St<double, 5> u = limited(li, lj, lk, s);
        const int p = didx(li, lj, lk);
        const unsigned char f = flg[p];
        if ((f & 64) && !(f & (1 << s))) {
            St<double, 5> n;
#pragma unroll
            for (int q = 0; q < 5; ++q) n[q] = u[q] - D[q * ND + p];
            if (admissible3(e, n)) u = n;
        }
        return u;
    };

    double smax = 0.0;
    // ---- 3. faces and balance, one axis at a time (compile-time axis)
    auto sweep = [&](auto axis_c) {
        constexpr int AX = decltype(axis_c)::value;
        constexpr int Fd[3] = {TX + (AX == 0), TY + (AX == 1), TZ + (AX == 2)};
        constexpr int nF = Fd[0] * Fd[1] * Fd[2];
        const int lo_side = 2 * AX, hi_side = lo_side + 1;
        const bool wall_lo = a.bc.type[lo_side] == kBcWall || a.bc.type[lo_side] == kBcNoSlip || a.bc.type[lo_side] == kBcMovingWall;
        const bool wall_hi = a.bc.type[hi_side] == kBcWall || a.bc.type[hi_side] == kBcNoSlip || a.bc.type[hi_side] == kBcMovingWall;
        for (int f = tid; f < nF; f += NT) {
            const int f3[3] = {f % Fd[0], (f / Fd[0]) % Fd[1], f / (Fd[0] * Fd[1])};
            const int g3[3] = {o3[0] + f3[0], o3[1] + f3[1], o3[2] + f3[2]};
            bool inside = true;
#pragma unroll
            for (int x = 0; x < 3; ++x) inside = inside && (x == AX ? g3[x] <= n3[x] : g3[x] < n3[x]);
            St<double, 5> F;
#pragma unroll
            for (int q = 0; q < 5; ++q) F[q] = 0.0;
            if (inside) {
                int L[3] = {f3[0], f3[1], f3[2]};
                L[AX] -= 1;
                const int t = g3[AX];
                St<double, 5> UL = predicted(L[0], L[1], L[2], hi_side), UR = predicted(f3[0], f3[1], f3[2], lo_side);
                if (t == 0) {
                    if (wall_lo)
                        UL = ghost_state(e, a.bc, lo_side, UR);
                    else if (a.bc.halo[lo_side] == kHaloNone)
                        UL = round_trip(e, side_ghost<5, FULL>(m, a.bc, e, a.U, lo_side, g3[0], g3[1], g3[2]));
                }
                if (t == n3[AX]) {
                    int c3[3] = {g3[0], g3[1], g3[2]};
                    c3[AX] = n3[AX] - 1;
                    if (wall_hi)
                        UR = ghost_state(e, a.bc, hi_side, UL);
                    else if (a.bc.halo[hi_side] == kHaloNone)
                        UR = round_trip(e, side_ghost<5, FULL>(m, a.bc, e, a.U, hi_side, c3[0], c3[1], c3[2]));
                }
                const double s = face_flux<RIEMANN>(e, a.shock_blend, UL, UR, AX, F);
                if (s > smax) smax = s;
            }
#pragma unroll
            for (int q = 0; q < 5; ++q) Fl[q * S::NF + f] = F[q];
        }
        __syncthreads();
        const double A = m.area[AX];
        for (int c = tid; c < NC; c += NT) {
            const int c3[3] = {c % TX, (c / TX) % TY, c / (TX * TY)};
            const int fl = (c3[2] * Fd[1] + c3[1]) * Fd[0] + c3[0];
            const int fr = fl + (AX == 0 ? 1 : (AX == 1 ? Fd[0] : Fd[0] * Fd[1]));
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double dd = Fl[q * S::NF + fr] * A - Fl[q * S::NF + fl] * A;
                acc[q * NC + c] = AX == 0 ? 0.0 - dd : acc[q * NC + c] - dd;
            }
        }
        __syncthreads();
    };
    sweep(std::integral_constant<int, 0>{});
    sweep(std::integral_constant<int, 1>{});
    sweep(std::integral_constant<int, 2>{});
    // ---- 4. the residual and the update
    const double dt = a.ctl->dt;
    for (int c = tid; c < NC; c += NT) {
        const int g3[3] = {o3[0] + c % TX, o3[1] + (c / TX) % TY, o3[2] + c / (TX * TY)};
        if (g3[0] >= m.nx || g3[1] >= m.ny || g3[2] >= m.nz) continue;
        const long long cell = cell_of(g3[0], g3[1], g3[2]);
        St<double, 5> r;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            r[q] = acc[q * NC + c] * m.inv_cell;
            if (a.Rv) r[q] = r[q] + a.Rv[q * m.plane + cell];
        }
        if (FULL && (a.bc.grav_on || a.bc.src)) {
            const St<double, 5> src = body_source<5>(a.bc, a.U, m.plane, cell);
#pragma unroll
            for (int q = 0; q < 5; ++q) r[q] = r[q] + src[q];
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const long long x = q * m.plane + cell;
            a.out[x] = a.mode == 0 ? r[q] : a.U[x] + dt * r[q];
        }
    }
    const double bm = block_max<NT>(smax, red);
    if (tid == 0) a.blockmax[b] = bm;
}

}   // namespace fvg
