// flux_quadrature = fourth: the residual with fourth-order face fluxes (fourth_order_fluxes and
// MusclReconstruction::reconstruct_conserved, cpp/src/Schemes.cpp:1202-1350, 1954-2133; the balance of
// Simulation::assemble, cpp/src/Simulation.cpp:1023-1036, 1290-1305), as face passes over arrays in HBM:
//
//   recon   WENO3-Z / WENO5-Z of the conserved cell averages at every face with a full stencil (a face of a side without a
//           halo keeps the side's first-order states, BoundaryManager::apply_side); a face whose states are not positive,
//           or whose density or pressure leaves the range of its stencil cells widened by its own width, takes the two
//           cells next to it. `good`: a full stencil, positive states and a quiet shock sensor.
//   point   the face averages turned into point values at the face centre, AL = UL - (sum over transverse axes of the
//           second difference of UL) / 24, where the face and its transverse neighbours (wrapped on a periodic axis) are
//           good and the result is positive (`pt`); else the averages.
//   flux    Fp = the Riemann flux of (AL, AR) at every face, and the per-CTA largest wave speed.
//   correct F = Fp + (the transverse second differences of Fp) / 24 where the face and its transverse neighbours have
//           point values; the flux of the averages where only the face has; else Fp.
//   balance the cell balance of F, the viscous residual, the body force and the sources, and the stage update.
//
// Faces of axis a form the lattice (nx + [a = 0]) x (ny + [a = 1]) x (nz + [a = 2]), index (k ey + j) ex + i, one array
// per conserved variable (NV of them: rho w is not held on a 2-D mesh, where the reference's is +0 on every face).
#pragma once

#include "stage.cuh"

namespace fvg {

struct FourthArgs {
    Mesh m;
    Bc bc;
    Eos<double> eos;
    double shock_blend, weno_eps;
    int periodic[3];           // both sides of the axis periodic (the transverse neighbours wrap)
    long long nf[3];           // faces per axis
    // per axis: NV planes of nf[a] values each
    double *UL[3], *UR[3], *AL[3], *AR[3], *Fp[3], *F[3];
    unsigned char *good[3], *pt[3], *full[3];
    const double* U;           // the state the residual is taken of
    // the stage update (StageArgs' meaning)
    int mode;
    double ca, cb;
    const double* U0;
    double* out;
    const double* Rv;
    double* blockmax;          // per-CTA largest wave speed of the flux pass (its grid is the stage's CTA count)
    const Ctl* ctl;
    const int* gate;
};

__device__ __forceinline__ void face_lattice(const Mesh& m, int a, long long f, int c[3], int e[3]) {
    e[0] = m.nx + (a == 0);
    e[1] = m.ny + (a == 1);
    e[2] = m.nz + (a == 2);
    c[0] = (int)(f % e[0]);
    c[1] = (int)((f / e[0]) % e[1]);
    c[2] = (int)(f / ((long long)e[0] * e[1]));
}

// the neighbour of face f at +-1 along transverse axis t (wrapped on a periodic axis; -1 beyond another side)
__device__ __forceinline__ long long face_nbr(const FourthArgs& a, long long f, const int c[3], const int e[3], int t, int s) {
    const int dims[3] = {a.m.nx, a.m.ny, a.m.nz};
    const long long st = t == 0 ? 1 : (t == 1 ? (long long)e[0] : (long long)e[0] * e[1]);
    const int ct = c[t] + s;
    if (ct >= 0 && ct < dims[t]) return f + s * st;
    if (!a.periodic[t]) return -1;
    return f - (long long)s * (dims[t] - 1) * st;
}

template <int NV> __device__ __forceinline__ double cons_m2(const St<double, NV>& u) {
    double r = u[1] * u[1] + u[2] * u[2];
    if constexpr (NV == 5) r = r + u[4] * u[4];
    return r;
}
// positive density and pressure without a division: rho > 0 and g1 (E rho - m^2 / 2) > gp rho
template <int NV> __device__ __forceinline__ bool cons_positive(double g1, double gp, const St<double, NV>& u) {
    return u[0] > 0.0 && g1 * (u[3] * u[0] - 0.5 * cons_m2<NV>(u)) > gp * u[0];
}
template <int NV> __device__ __forceinline__ double cons_pressure(double g1, double gp, const St<double, NV>& u) {
    return g1 * (u[3] - 0.5 * cons_m2<NV>(u) / u[0]) - gp;
}

template <int NV> __device__ __forceinline__ St<double, NV> load_face(const double* p, long long nf, long long f) {
    St<double, NV> u;
#pragma unroll
    for (int q = 0; q < NV; ++q) u[q] = p[q * nf + f];
    return u;
}
template <int NV> __device__ __forceinline__ void store_face(double* p, long long nf, long long f, const St<double, NV>& u) {
#pragma unroll
    for (int q = 0; q < NV; ++q) p[q * nf + f] = u[q];
}

// ---- recon: the conserved reconstruction of axis A's faces and their `good` flags (ConservedLines::line and the first
// loop of fourth_order_fluxes)
template <int DIM, int NV, int A, bool FIVE>
__global__ void __launch_bounds__(256) k4_recon(const FourthArgs a) {
    if (!*a.gate) return;
    const Mesh& m = a.m;
    const double g1 = a.eos.gamma - 1.0, gp = a.eos.type == kIdeal ? 0.0 : a.eos.gamma * a.eos.p_inf;
    const int dims[3] = {m.nx, m.ny, m.nz};
    const bool has_lo = a.bc.halo[2 * A] != kHaloNone, has_hi = a.bc.halo[2 * A + 1] != kHaloNone;
    const long long nf = a.nf[A];
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
        int c[3], e[3];
        face_lattice(m, A, f, c, e);
        const int ca = c[A], n_a = dims[A];
        St<double, NV> ul, ur;
        const bool full_stencil = (ca > 0 && ca < n_a) || (ca == 0 && has_lo) || (ca == n_a && has_hi);
        if (!full_stencil) {   // apply_side's states: the cell next to the side and its ghost
            int cell[3] = {c[0], c[1], c[2]};
            if (ca == n_a) cell[A] = n_a - 1;
            side_states<NV>(m, a.bc, a.eos, a.U, 2 * A + (ca == n_a ? 1 : 0), cell[0], cell[1], cell[2], ul, ur);
        } else {
            // the stencil cells (padded positions ca - 3 .. ca + 2, or ca - 2 .. ca + 1), conserved
            constexpr int ncell = FIVE ? 6 : 4;
            const int first = ca - (FIVE ? 3 : 2);
            St<double, NV> s[ncell];
#pragma unroll
            for (int l = 0; l < ncell; ++l) {
                int p[3] = {c[0], c[1], c[2]};
                p[A] = first + l;
                s[l] = stencil_cons<DIM, NV>(m, a.bc, a.eos, a.U, p[0], p[1], DIM == 3 ? p[2] : 0);
            }
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                if constexpr (FIVE) {
                    ul[q] = weno5z(s[0][q], s[1][q], s[2][q], s[3][q], s[4][q], a.weno_eps);
                    ur[q] = weno5z(s[5][q], s[4][q], s[3][q], s[2][q], s[1][q], a.weno_eps);
                } else {
                    ul[q] = weno3z(s[0][q], s[1][q], s[2][q], a.weno_eps);
                    ur[q] = weno3z(s[3][q], s[2][q], s[1][q], a.weno_eps);
                }
            }
            // admissible: positive, density and pressure inside the stencil cells' range widened by its own width
            bool ok = cons_positive<NV>(g1, gp, ul) && cons_positive<NV>(g1, gp, ur);
            if (ok) {
                double rlo = 1e300, rhi = -1e300, plo = 1e300, phi = -1e300;
#pragma unroll
                for (int l = 0; l < ncell; ++l) {
                    const double pc = cons_pressure<NV>(g1, gp, s[l]);
                    rlo = vmin(rlo, s[l][0]);
                    rhi = vmax(rhi, s[l][0]);
                    plo = vmin(plo, pc);
                    phi = vmax(phi, pc);
                }
                const double rw = rhi - rlo, pw = phi - plo;
                rlo -= rw;
                rhi += rw;
                plo -= pw;
                phi += pw;
                const double pfl = cons_pressure<NV>(g1, gp, ul), pfr = cons_pressure<NV>(g1, gp, ur);
                ok = ok && ul[0] >= rlo && ul[0] <= rhi && pfl >= plo && pfl <= phi;
                ok = ok && ur[0] >= rlo && ur[0] <= rhi && pfr >= plo && pfr <= phi;
            }
            if (!ok) {
                constexpr int left = FIVE ? 2 : 1;
                ul = s[left];
                ur = s[left + 1];
            }
        }
        store_face<NV>(a.UL[A], nf, f, ul);
        store_face<NV>(a.UR[A], nf, f, ur);
        bool good = full_stencil && cons_positive<NV>(g1, gp, ul) && cons_positive<NV>(g1, gp, ur);
        if (good && a.shock_blend > 0.0) {
            const double pL = cons_pressure<NV>(g1, gp, ul), pR = cons_pressure<NV>(g1, gp, ur);
            if (fabs(pR - pL) > a.shock_blend * vmin(pL, pR)) good = false;
        }
        a.good[A][f] = good ? 1 : 0;
    }
}

// ---- point: the point values of axis A's faces (the second loop of fourth_order_fluxes)
template <int DIM, int NV, int A>
__global__ void __launch_bounds__(256) k4_point(const FourthArgs a) {
    if (!*a.gate) return;
    const double g1 = a.eos.gamma - 1.0, gp = a.eos.type == kIdeal ? 0.0 : a.eos.gamma * a.eos.p_inf;
    const long long nf = a.nf[A];
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
        const St<double, NV> ul = load_face<NV>(a.UL[A], nf, f), ur = load_face<NV>(a.UR[A], nf, f);
        St<double, NV> al = ul, ar = ur;
        unsigned char pt = 0;
        if (a.good[A][f]) {
            int c[3], e[3];
            face_lattice(a.m, A, f, c, e);
            long long nb[2][2];
            int cnt = 0;
            bool ok = true;
#pragma unroll
            for (int t = 0; t < DIM; ++t) {
                if (t == A || !ok) continue;
                nb[cnt][0] = face_nbr(a, f, c, e, t, -1);
                nb[cnt][1] = face_nbr(a, f, c, e, t, 1);
                ok = nb[cnt][0] >= 0 && nb[cnt][1] >= 0 && a.good[A][nb[cnt][0]] && a.good[A][nb[cnt][1]];
                ++cnt;
            }
            if (ok) {
                St<double, NV> pl = ul, pr = ur;
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    double dl = 0.0, dr = 0.0;
                    for (int u = 0; u < cnt; ++u) {
                        dl += a.UL[A][q * nf + nb[u][1]] - 2.0 * ul[q] + a.UL[A][q * nf + nb[u][0]];
                        dr += a.UR[A][q * nf + nb[u][1]] - 2.0 * ur[q] + a.UR[A][q * nf + nb[u][0]];
                    }
                    pl[q] -= dl / 24.0;
                    pr[q] -= dr / 24.0;
                }
                if (cons_positive<NV>(g1, gp, pl) && cons_positive<NV>(g1, gp, pr)) {
                    al = pl;
                    ar = pr;
                    pt = 1;
                }
            }
        }
        store_face<NV>(a.AL[A], nf, f, al);
        store_face<NV>(a.AR[A], nf, f, ar);
        a.pt[A][f] = pt;
    }
}

// ---- flux: `full` flags, the Riemann flux of the point values (or averages) and the per-CTA largest wave speed of all
// axes' faces (RiemannSolver::compute_flux); the grid is the stage's CTA count, each CTA writes blockmax[blockIdx.x]
template <int DIM, int NV, int RIEMANN>
__global__ void __launch_bounds__(256) k4_flux(const FourthArgs a) {
    __shared__ double red[32];
    if (!*a.gate) return;
    double smax = 0.0;
#pragma unroll 1
    for (int A = 0; A < DIM; ++A) {
        const long long nf = a.nf[A];
        for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
            unsigned char full = 0;
            if (a.pt[A][f]) {
                int c[3], e[3];
                face_lattice(a.m, A, f, c, e);
                bool ok = true;
                for (int t = 0; t < DIM && ok; ++t) {
                    if (t == A) continue;
                    const long long g0 = face_nbr(a, f, c, e, t, -1), g1 = face_nbr(a, f, c, e, t, 1);
                    ok = g0 >= 0 && g1 >= 0 && a.pt[A][g0] && a.pt[A][g1];
                }
                full = ok ? 1 : 0;
            }
            a.full[A][f] = full;
            St<double, NV> fl;
            const double s = face_flux<RIEMANN>(a.eos, a.shock_blend, load_face<NV>(a.AL[A], nf, f), load_face<NV>(a.AR[A], nf, f), A, fl);
            if (s > smax) smax = s;
            store_face<NV>(a.Fp[A], nf, f, fl);
        }
    }
    const double bm = block_max<256>(smax, red);
    if (threadIdx.x == 0) a.blockmax[blockIdx.x] = bm;
}

// ---- correct: the fourth-order flux of axis A's faces (the last loop of fourth_order_fluxes)
template <int DIM, int NV, int RIEMANN, int A>
__global__ void __launch_bounds__(256) k4_correct(const FourthArgs a) {
    if (!*a.gate) return;
    const long long nf = a.nf[A];
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
        const St<double, NV> fp = load_face<NV>(a.Fp[A], nf, f);
        St<double, NV> out = fp;
        if (a.full[A][f]) {
            int c[3], e[3];
            face_lattice(a.m, A, f, c, e);
            long long nb[2][2];
            int cnt = 0;
#pragma unroll
            for (int t = 0; t < DIM; ++t) {
                if (t == A) continue;
                nb[cnt][0] = face_nbr(a, f, c, e, t, -1);
                nb[cnt][1] = face_nbr(a, f, c, e, t, 1);
                ++cnt;
            }
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                double d = 0.0;
                for (int u = 0; u < cnt; ++u) d += a.Fp[A][q * nf + nb[u][1]] - 2.0 * fp[q] + a.Fp[A][q * nf + nb[u][0]];
                out[q] = fp[q] + d / 24.0;
            }
        } else if (a.pt[A][f]) {   // a point value without the full correction: the flux of the averaged states
            face_flux<RIEMANN>(a.eos, a.shock_blend, load_face<NV>(a.UL[A], nf, f), load_face<NV>(a.UR[A], nf, f), A, out);
        }
        store_face<NV>(a.F[A], nf, f, out);
    }
}

// ---- balance: R of every cell from the face fluxes, then the viscous residual, the body force, the sources and the
// stage update (the epilogue of the stage kernel)
template <int DIM, int NV>
__global__ void __launch_bounds__(256) k4_balance(const FourthArgs a) {
    if (!*a.gate) return;
    const Mesh& m = a.m;
    const double dt = a.ctl->dt;
    for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < m.ncells; cell += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(cell % m.nx), j = (int)((cell / m.nx) % m.ny), k = (int)(cell / ((long long)m.nx * m.ny));
        const long long fx = ((long long)k * m.ny + j) * (m.nx + 1) + i;
        const long long fy = ((long long)k * (m.ny + 1) + j) * m.nx + i;
        const long long fz = ((long long)k * m.ny + j) * m.nx + i;
        St<double, NV> r;
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const double* Fx = a.F[0] + q * a.nf[0];
            const double* Fy = a.F[1] + q * a.nf[1];
            double v = (0.0 - (Fx[fx + 1] * m.area[0] - Fx[fx] * m.area[0])) - (Fy[fy + m.nx] * m.area[1] - Fy[fy] * m.area[1]);
            if constexpr (DIM == 3) {
                const double* Fz = a.F[2] + q * a.nf[2];
                v = v - (Fz[fz + (long long)m.nx * m.ny] * m.area[2] - Fz[fz] * m.area[2]);
            }
            r[q] = v * m.inv_cell;
            if (a.Rv) r[q] = r[q] + a.Rv[q * m.plane + cell];
        }
        if (a.bc.grav_on) add_body_force<NV>(a.bc, read_state<NV>(a.bc, a.U, m.plane, cell), r);
        if (a.bc.src) add_source<NV>(a.bc, m.plane, cell, r);
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const long long x = q * m.plane + cell;
            a.out[x] = a.mode == kStoreR ? r[q] : (a.mode == kAxpy ? a.U[x] + dt * r[q] : a.ca * a.U0[x] + a.cb * (a.U[x] + dt * r[q]));
        }
    }
}

}   // namespace fvg
