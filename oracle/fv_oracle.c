/* CPU restatement of the reference's uniform-grid finite-volume right-hand side and time step. TEST
 * INFRASTRUCTURE (see fv_oracle.h): the checker of the CUDA path, never part of it.
 *
 * Build: gcc -O2 -std=c11 -fPIC -shared -fno-fast-math -ffp-contract=off (the reference's floating-point
 * contract, cpp/CMakeLists.txt:85: no contraction into fused multiply-adds, IEEE division and square root). The
 * operation order of every expression is the reference's; file:line citations are to the reference tree. */
#include "fv_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NV 5
typedef double St[NV];

/* std::max / std::min semantics (the reference headers use them): max(a, b) = a < b ? b : a, min(a, b) = b < a ? b : a */
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static const int kMom[3] = {1, 2, 4};
static const double kEosEps = 1e-10;   /* Core.hpp:169 */
static const double kDenomEps = 1e-14; /* Schemes.cpp:64 */
static const double kMachEps = 1e-12;  /* Schemes.cpp:66 */
static const double kDtEps = 1e-10;    /* TimeScheme.cpp:19 */

/* ---------------------------------------------------------------- EOS (Core.hpp:173-238) */
typedef struct {
    int type;
    double gamma, p_inf;
} Eos;

static void p2c(const Eos* e, const double* W, double* U) {
    const double rho = W[0], u = W[1], v = W[2], p = W[3], w = W[4];
    const double ke = 0.5 * rho * (u * u + v * v + w * w);
    const double en = e->type == ORC_IDEAL ? p / (e->gamma - 1.0) : (p + e->gamma * e->p_inf) / (e->gamma - 1.0);
    U[0] = rho;
    U[1] = rho * u;
    U[2] = rho * v;
    U[3] = en + ke;
    U[4] = rho * w;
}

static void c2p(const Eos* e, const double* U, double* W, double* inv_rho) {
    const double rho = dmax(U[0], kEosEps);
    const double inv = 1.0 / rho;
    if (inv_rho) *inv_rho = inv;
    const double u = U[1] * inv, v = U[2] * inv, w = U[4] * inv;
    const double e_kin = 0.5 * rho * (u * u + v * v + w * w);
    const double rho_e = U[3] - e_kin;
    const double p = e->type == ORC_IDEAL ? (e->gamma - 1.0) * rho_e : (e->gamma - 1.0) * rho_e - e->gamma * e->p_inf;
    W[0] = rho;
    W[1] = u;
    W[2] = v;
    W[3] = dmax(p, kEosEps);
    W[4] = w;
}

static double sound_speed_inv(const Eos* e, double p, double inv_rho) {
    if (e->type == ORC_IDEAL) return sqrt(e->gamma * dmax(p, kEosEps) * inv_rho);
    return sqrt(e->gamma * (p + e->p_inf) * inv_rho);
}

static double sound_speed(const Eos* e, double p, double rho) {
    if (e->type == ORC_IDEAL) return sqrt(e->gamma * dmax(p, kEosEps) / dmax(rho, kEosEps));
    return sqrt(e->gamma * (p + e->p_inf) / dmax(rho, kEosEps));
}

static void round_trip(const Eos* e, double* U) {
    St W;
    c2p(e, U, W, NULL);
    p2c(e, W, U);
}

/* ---------------------------------------------------------------- Riemann solvers (Schemes.cpp:104-229) */
static inline double safe_denom(double x) { return copysign(dmax(fabs(x), kDenomEps), x); }

static double hllc_core(const double* WL, const double* WR, const double* UL, const double* UR, double inv_L, double inv_R, double c_L,
                        double c_R, int axis, double shock_blend, double* F) {
    const double rho_L = WL[0], p_L = WL[3];
    const double rho_R = WR[0], p_R = WR[3];
    const double vel_L[3] = {WL[1], WL[2], WL[4]};
    const double vel_R[3] = {WR[1], WR[2], WR[4]};
    const double E_L = UL[3] * inv_L, E_R = UR[3] * inv_R;
    const double Vn_L = vel_L[axis], Vn_R = vel_R[axis];
    const int mn = kMom[axis];
    St FL, FR;
    FL[0] = rho_L * Vn_L;
    FR[0] = rho_R * Vn_R;
    for (int a = 0; a < 3; ++a) {
        FL[kMom[a]] = rho_L * vel_L[a] * Vn_L;
        FR[kMom[a]] = rho_R * vel_R[a] * Vn_R;
    }
    FL[mn] = FL[mn] + p_L;
    FR[mn] = FR[mn] + p_R;
    FL[3] = Vn_L * (rho_L * E_L + p_L);
    FR[3] = Vn_R * (rho_R * E_R + p_R);
    const double S_L = dmin(Vn_L - c_L, Vn_R - c_R);
    const double S_R = dmax(Vn_L + c_L, Vn_R + c_R);
    const double num = rho_R * Vn_R * (S_R - Vn_R) - rho_L * Vn_L * (S_L - Vn_L) + p_L - p_R;
    const double den = rho_R * (S_R - Vn_R) - rho_L * (S_L - Vn_L);
    const double S_M = num / safe_denom(den);
    const double den_star_L = safe_denom(S_L - S_M);
    const double den_star_R = safe_denom(S_R - S_M);
    const double den_pL = safe_denom(S_L - Vn_L);
    const double den_pR = safe_denom(S_R - Vn_R);
    const double fL = rho_L * (S_L - Vn_L) / den_star_L;
    const double fR = rho_R * (S_R - Vn_R) / den_star_R;
    St UsL, UsR;
    UsL[0] = fL;
    UsR[0] = fR;
    for (int a = 0; a < 3; ++a) {
        UsL[kMom[a]] = fL * (a == axis ? S_M : vel_L[a]);
        UsR[kMom[a]] = fR * (a == axis ? S_M : vel_R[a]);
    }
    UsL[3] = fL * (E_L + (S_M - Vn_L) * (S_M + p_L / (rho_L * den_pL)));
    UsR[3] = fR * (E_R + (S_M - Vn_R) * (S_M + p_R / (rho_R * den_pR)));
    for (int q = 0; q < NV; ++q) F[q] = 0.0;
    if (S_L >= 0)
        for (int q = 0; q < NV; ++q) F[q] = FL[q];
    if (S_L < 0 && S_M >= 0)
        for (int q = 0; q < NV; ++q) F[q] = FL[q] + S_L * (UsL[q] - UL[q]);
    if (S_M < 0 && S_R >= 0)
        for (int q = 0; q < NV; ++q) F[q] = FR[q] + S_R * (UsR[q] - UR[q]);
    if (S_R < 0)
        for (int q = 0; q < NV; ++q) F[q] = FR[q];
    if (shock_blend > 0.0) {
        const double s = fabs(p_R - p_L) / dmin(p_L, p_R);
        if (s > shock_blend) {
            const double phi = dmin((s - shock_blend) / shock_blend, 1.0);
            St Fh;
            if (S_L >= 0) {
                for (int q = 0; q < NV; ++q) Fh[q] = FL[q];
            } else if (S_R <= 0) {
                for (int q = 0; q < NV; ++q) Fh[q] = FR[q];
            } else {
                const double inv = 1.0 / (S_R - S_L);
                for (int q = 0; q < NV; ++q) Fh[q] = (S_R * FL[q] - S_L * FR[q] + S_L * S_R * (UR[q] - UL[q])) * inv;
            }
            for (int q = 0; q < NV; ++q) F[q] = (1.0 - phi) * F[q] + phi * Fh[q];
        }
    }
    return dmax(fabs(S_L), fabs(S_R));
}

typedef struct {
    Eos eos;
    int type;
    double shock_blend;
} Riemann;

/* RiemannSolver::face_flux (Schemes.cpp:202-208) with hllc (:108-113) and lowmach_flux (:213-229) */
static double face_flux(const Riemann* rs, const double* UL, const double* UR, int axis, double* F) {
    double inv_L, inv_R;
    St WL, WR;
    c2p(&rs->eos, UL, WL, &inv_L);
    c2p(&rs->eos, UR, WR, &inv_R);
    if (rs->type != ORC_LOWMACH)
        return hllc_core(WL, WR, UL, UR, inv_L, inv_R, sound_speed_inv(&rs->eos, WL[3], inv_L), sound_speed_inv(&rs->eos, WR[3], inv_R), axis,
                         rs->shock_blend, F);
    const double c_L = sound_speed_inv(&rs->eos, WL[3], inv_L);
    const double c_R = sound_speed_inv(&rs->eos, WR[3], inv_R);
    const double M_L = sqrt(WL[1] * WL[1] + WL[2] * WL[2] + WL[4] * WL[4]) / (c_L + kMachEps);
    const double M_R = sqrt(WR[1] * WR[1] + WR[2] * WR[2] + WR[4] * WR[4]) / (c_R + kMachEps);
    const double z = dmin(dmax(dmax(M_L, M_R), 1e-4), 1.0);
    for (int a = 0; a < 3; ++a) {
        const int m = kMom[a];
        const double avg = 0.5 * (WL[m] + WR[m]);
        const double half = 0.5 * (WL[m] - WR[m]);
        WL[m] = avg + z * half;
        WR[m] = avg - z * half;
    }
    St UsL, UsR;
    p2c(&rs->eos, WL, UsL);
    p2c(&rs->eos, WR, UsR);
    return hllc_core(WL, WR, UsL, UsR, inv_L, inv_R, c_L, c_R, axis, rs->shock_blend, F);
}

/* ---------------------------------------------------------------- limiters and WENO-Z (Schemes.hpp:93-117, Schemes.cpp:328-353) */
static inline double sgn(double x) { return (x > 0.0) ? 1.0 : ((x < 0.0) ? -1.0 : 0.0); }
static double apply_limiter(int l, double a, double b) {
    switch (l) {
    case ORC_MINMOD: return 0.5 * (sgn(a) + sgn(b)) * dmin(fabs(a), fabs(b));
    case ORC_VANLEER: {
        const double ab = a * b;
        return (ab > 0) ? 2.0 * ab / (a + b) : 0.0;
    }
    case ORC_MC:
        if (!(a * b > 0)) return 0.0;
        return dmin(dmin(2.0 * fabs(a), 0.5 * fabs(a + b)), 2.0 * fabs(b)) * sgn(a);
    default:
        if (!(a * b > 0)) return 0.0;
        return fmin(fmin(2.0 * fabs(a), fabs(2.0 * a + b) / 3.0), 2.0 * fabs(b)) * sgn(a);
    }
}

static double weno3z(double c0, double c1, double c2, double eps_rel) {
    const double eps = eps_rel * (c0 * c0 + c1 * c1 + c2 * c2) * (1.0 / 3.0) + 1e-300;
    const double v0 = -0.5 * c0 + 1.5 * c1, v1 = 0.5 * c1 + 0.5 * c2;
    const double b0 = (c1 - c0) * (c1 - c0), b1 = (c2 - c1) * (c2 - c1);
    const double tau = fabs(b0 - b1);
    const double a0 = (1.0 / 3.0) * (1.0 + tau / (b0 + eps)), a1 = (2.0 / 3.0) * (1.0 + tau / (b1 + eps));
    return (a0 * v0 + a1 * v1) / (a0 + a1);
}

static double weno5z(double c0, double c1, double c2, double c3, double c4, double eps_rel) {
    const double eps = eps_rel * (c0 * c0 + c1 * c1 + c2 * c2 + c3 * c3 + c4 * c4) * 0.2 + 1e-300;
    const double p0 = (2.0 * c0 - 7.0 * c1 + 11.0 * c2) / 6.0;
    const double p1 = (-c1 + 5.0 * c2 + 2.0 * c3) / 6.0;
    const double p2 = (2.0 * c2 + 5.0 * c3 - c4) / 6.0;
    const double s0 = c0 - 2.0 * c1 + c2, t0 = c0 - 4.0 * c1 + 3.0 * c2;
    const double s1 = c1 - 2.0 * c2 + c3, t1 = c1 - c3;
    const double s2 = c2 - 2.0 * c3 + c4, t2 = 3.0 * c2 - 4.0 * c3 + c4;
    const double b0 = (13.0 / 12.0) * s0 * s0 + 0.25 * t0 * t0;
    const double b1 = (13.0 / 12.0) * s1 * s1 + 0.25 * t1 * t1;
    const double b2 = (13.0 / 12.0) * s2 * s2 + 0.25 * t2 * t2;
    const double tau = fabs(b0 - b2);
    const double a0 = 0.1 * (1.0 + tau / (b0 + eps)), a1 = 0.6 * (1.0 + tau / (b1 + eps)), a2 = 0.3 * (1.0 + tau / (b2 + eps));
    return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}

/* ---------------------------------------------------------------- mesh and boundaries */
typedef struct {
    const orc_config* c;
    Eos eos;
    Riemann rs;
    int nx, ny, nz, three_d;
    double dx, dy, dz;
} Ctx;

static void ctx_init(Ctx* x, const orc_config* c) {
    x->c = c;
    x->eos.type = c->eos;
    x->eos.gamma = c->gamma;
    x->eos.p_inf = c->p_inf;
    x->rs.eos = x->eos;
    x->rs.type = c->riemann;
    x->rs.shock_blend = c->shock_blend;
    x->nx = c->nx;
    x->ny = c->ny;
    x->nz = c->nz;
    x->three_d = c->nz > 1;
    x->dx = c->Lx / c->nx;
    x->dy = c->Ly / c->ny;
    x->dz = c->Lz / c->nz; /* generate_cartesian_mesh_3d (Core.cpp:20-40); 2-D: nz = 1 */
}

static inline size_t cell(const Ctx* x, int i, int j, int k) { return ((size_t)k * x->ny + j) * x->nx + i; }

/* BoundaryManager::ghost_state (Boundaries.cpp:106-153); u_target: the mass-flow inlet velocity of the side */
static void ghost_state(const Ctx* x, int side, const double* Ui, double u_target, double* Ug) {
    const int bc = x->c->bc[side];
    if (bc == ORC_TRANSMISSIVE) {
        memcpy(Ug, Ui, sizeof(St));
        return;
    }
    const int axis = side / 2;
    const double nxn = axis == 0 ? 1.0 : 0.0, nyn = axis == 1 ? 1.0 : 0.0, nzn = axis == 2 ? 1.0 : 0.0;
    St Wi, Wg;
    c2p(&x->eos, Ui, Wi, NULL);
    memcpy(Wg, Wi, sizeof(St));
    switch (bc) {
    case ORC_WALL: {
        const double Vn = Wi[1] * nxn + Wi[2] * nyn + Wi[4] * nzn;
        Wg[1] = Wi[1] - 2.0 * Vn * nxn;
        Wg[2] = Wi[2] - 2.0 * Vn * nyn;
        Wg[4] = Wi[4] - 2.0 * Vn * nzn;
        break;
    }
    case ORC_NOSLIP:
        Wg[1] = -Wi[1];
        Wg[2] = -Wi[2];
        Wg[4] = -Wi[4];
        break;
    case ORC_MOVINGWALL:
    case ORC_VELINLET:
        Wg[1] = 2.0 * x->c->u_in - Wi[1];
        Wg[2] = 2.0 * x->c->v_in - Wi[2];
        Wg[4] = -Wi[4];
        break;
    case ORC_MASSFLOWINLET:
        Wg[1] = 2.0 * u_target - Wi[1];
        Wg[2] = 2.0 * x->c->v_in - Wi[2];
        Wg[4] = -Wi[4];
        break;
    case ORC_OUTLET: {
        const double Vn = Wi[1] * nxn + Wi[2] * nyn + Wi[4] * nzn;
        const int outflow = Vn >= 0;
        Wg[1] = outflow ? Wi[1] : 0.0;
        Wg[2] = outflow ? Wi[2] : 0.0;
        Wg[4] = outflow ? Wi[4] : 0.0;
        Wg[3] = dmax(x->c->p_out, 1e-5);
        break;
    }
    default: break;
    }
    p2c(&x->eos, Wg, Ug);
}

static int n_axis(const Ctx* x, int a) { return a == 0 ? x->nx : (a == 1 ? x->ny : x->nz); }

/* The mass-flow inlet velocity of a side (BoundaryManager::apply_side, Boundaries.cpp:285-293): the side's mean density in
 * boundary-face order k = 0 .. n-1 (Core.hpp boundary_cell). */
static double u_target_of(const Ctx* x, const double* U, int side) {
    if (x->c->bc[side] != ORC_MASSFLOWINLET) return 0.0;
    const int axis = side / 2, hi = side & 1;
    double sum = 0.0;
    int count = 0;
    const int nt0 = axis == 0 ? x->ny : x->nx, nt1 = axis == 2 ? x->ny : x->nz;
    for (int b = 0; b < nt1; ++b)
        for (int a = 0; a < nt0; ++a) {
            int i, j, k;
            if (axis == 0) { i = hi ? x->nx - 1 : 0; j = a; k = b; }
            else if (axis == 1) { i = a; j = hi ? x->ny - 1 : 0; k = b; }
            else { i = a; j = b; k = hi ? x->nz - 1 : 0; }
            St W;
            c2p(&x->eos, U + NV * cell(x, i, j, k), W, NULL);
            sum += W[0];
            ++count;
        }
    const double rho_avg = dmax(sum / (double)count, 1e-5);
    return (x->c->rho_in * x->c->u_in) / rho_avg;
}

/* Which sides have a ghost layer `depth` deep (Simulation.cpp:868-905, 1107-1176): the periodic wrap of a periodic axis
 * (both sides periodic, at least `depth` cells), else with boundary_order = 2 the BC's ghost slab (not for periodic or
 * non-reflecting sides, and only with at least `depth` cells). 0 none, 1 wrap, 2 slab. */
static void halo_kinds(const Ctx* x, int depth, int kind[6]) {
    for (int s = 0; s < 6; ++s) kind[s] = 0;
    const int naxes = x->three_d ? 3 : 2;
    for (int a = 0; a < naxes; ++a) {
        const int per = x->c->bc[2 * a] == ORC_PERIODIC && x->c->bc[2 * a + 1] == ORC_PERIODIC;
        for (int h = 0; h < 2; ++h) {
            const int s = 2 * a + h, bt = x->c->bc[s];
            if (per && n_axis(x, a) >= depth)
                kind[s] = 1;
            else if (x->c->boundary_order == 2 && bt != ORC_PERIODIC && bt != ORC_NONREFLECTING && n_axis(x, a) >= depth)
                kind[s] = 2;
        }
    }
}

/* The conservative state of a cell outside the domain along axis `a` only (position p < 0 or >= n along it), the other
 * indices inside: the wrap-around cell, the ghost-slab state of the mirrored cell (fill_ghost_slab,
 * Boundaries.cpp:202-228: layer l from the boundary is ghost_state of the interior cell l cells from it), or the edge
 * cell (replication). */
static void outside_state(const Ctx* x, const double* U, const int kind[6], const double ut[6], int i, int j, int k, double* out) {
    int idx[3] = {i, j, k};
    const int n3[3] = {x->nx, x->ny, x->nz};
    int a = -1;
    for (int d = 0; d < 3; ++d)
        if (idx[d] < 0 || idx[d] >= n3[d]) a = (a < 0) ? d : 9;
    if (a < 0) {
        memcpy(out, U + NV * cell(x, i, j, k), sizeof(St));
        return;
    }
    if (a == 9) { /* outside along two axes: edge replication (pad_primitives) */
        for (int d = 0; d < 3; ++d) idx[d] = idx[d] < 0 ? 0 : (idx[d] >= n3[d] ? n3[d] - 1 : idx[d]);
        memcpy(out, U + NV * cell(x, idx[0], idx[1], idx[2]), sizeof(St));
        return;
    }
    const int hi = idx[a] >= n3[a];
    const int side = 2 * a + hi;
    if (kind[side] == 1) {
        idx[a] = hi ? idx[a] - n3[a] : idx[a] + n3[a];
        memcpy(out, U + NV * cell(x, idx[0], idx[1], idx[2]), sizeof(St));
    } else if (kind[side] == 2) {
        const int l = hi ? idx[a] - n3[a] : -1 - idx[a];
        idx[a] = hi ? n3[a] - 1 - l : l;
        ghost_state(x, side, U + NV * cell(x, idx[0], idx[1], idx[2]), ut[side], out);
    } else {
        idx[a] = hi ? n3[a] - 1 : 0;
        memcpy(out, U + NV * cell(x, idx[0], idx[1], idx[2]), sizeof(St));
    }
}

/* First-order face states of a boundary face (BoundaryManager::apply_side, Boundaries.cpp:277-373) */
static int side_states(const Ctx* x, const double* U, const double ut[6], int side, int i, int j, int k, double* UL, double* UR) {
    const int bc = x->c->bc[side];
    const double* Ui = U + NV * cell(x, i, j, k);
    St Ug;
    if (bc == ORC_PERIODIC) {
        int idx[3] = {i, j, k};
        const int a = side / 2, n = n_axis(x, a);
        idx[a] = (side & 1) ? idx[a] - (n - 1) : idx[a] + (n - 1);
        memcpy(Ug, U + NV * cell(x, idx[0], idx[1], idx[2]), sizeof(St));
    } else if (bc == ORC_NONREFLECTING) {
        return -2;
    } else {
        ghost_state(x, side, Ui, ut[side], Ug);
    }
    if (side & 1) {
        memcpy(UL, Ui, sizeof(St));
        memcpy(UR, Ug, sizeof(St));
    } else {
        memcpy(UL, Ug, sizeof(St));
        memcpy(UR, Ui, sizeof(St));
    }
    return 0;
}

/* ---------------------------------------------------------------- face states of the whole mesh */
/* Face arrays in the reference's face order (Core.hpp:116-120): x faces (k*ny + j)*(nx+1) + i, then y faces
 * (k*(ny+1) + j)*nx + i, then z faces (k*ny + j)*nx + i. */
typedef struct {
    size_t nxf, nyf, nzf, n;
} Faces;

static Faces faces_of(const Ctx* x) {
    Faces f;
    f.nxf = (size_t)(x->nx + 1) * x->ny * x->nz;
    f.nyf = (size_t)x->nx * (x->ny + 1) * x->nz;
    f.nzf = x->three_d ? (size_t)x->nx * x->ny * (x->nz + 1) : 0;
    f.n = f.nxf + f.nyf + f.nzf;
    return f;
}
static inline size_t xface(const Ctx* x, int i, int j, int k) { return ((size_t)k * x->ny + j) * (x->nx + 1) + i; }
static inline size_t yface(const Ctx* x, const Faces* f, int i, int j, int k) { return f->nxf + ((size_t)k * (x->ny + 1) + j) * x->nx + i; }
static inline size_t zface(const Ctx* x, const Faces* f, int i, int j, int k) { return f->nxf + f->nyf + ((size_t)k * x->ny + j) * x->nx + i; }
static size_t face_of(const Ctx* x, const Faces* f, int axis, int i, int j, int k) {
    return axis == 0 ? xface(x, i, j, k) : (axis == 1 ? yface(x, f, i, j, k) : zface(x, f, i, j, k));
}

/* The left / right states of every face: the reconstruction (MusclReconstruction::reconstruct / reconstruct_3d /
 * reconstruct_weno, Schemes.cpp:400-757) of the faces with a full stencil, the first-order states of the others (through the
 * conservative-primitive round trip when a reconstruction is on). */
static int face_states(const Ctx* x, const double* U, const double ut[6], double* UL, double* UR) {
    const orc_config* c = x->c;
    const Faces F = faces_of(x);
    const int recon = c->recon;
    const int pad = recon == ORC_WENO5 ? 3 : 2;
    int kind[6];
    halo_kinds(x, pad, kind);
    if (recon == ORC_FIRST_ORDER)
        for (int s = 0; s < 6; ++s) kind[s] = 0;
    const int naxes = x->three_d ? 3 : 2;
    const int planar = !x->three_d;
    for (int axis = 0; axis < naxes; ++axis) {
        const int na = n_axis(x, axis);
        const int ni = axis == 0 ? x->nx + 1 : x->nx, nj = axis == 1 ? x->ny + 1 : x->ny, nk = axis == 2 ? x->nz + 1 : x->nz;
        for (int k = 0; k < nk; ++k)
            for (int j = 0; j < nj; ++j)
                for (int i = 0; i < ni; ++i) {
                    const int t = axis == 0 ? i : (axis == 1 ? j : k);
                    const size_t f = face_of(x, &F, axis, i, j, k);
                    double* ul = UL + NV * f;
                    double* ur = UR + NV * f;
                    const int full = recon != ORC_FIRST_ORDER &&
                                     ((t > 0 && t < na) || (t == 0 && kind[2 * axis]) || (t == na && kind[2 * axis + 1]));
                    if (!full) {
                        int cc[3] = {i, j, k};
                        if (t == 0) {
                            if (t == na) return -3;
                        } else if (t == na) {
                            cc[axis] = na - 1;
                        } else { /* first order between two cells */
                            int cl[3] = {i, j, k};
                            cl[axis] = t - 1;
                            memcpy(ul, U + NV * cell(x, cl[0], cl[1], cl[2]), sizeof(St));
                            memcpy(ur, U + NV * cell(x, i, j, k), sizeof(St));
                            continue;
                        }
                        const int side = 2 * axis + (t == na);
                        if (side_states(x, U, ut, side, cc[0], cc[1], cc[2], ul, ur)) return -2;
                        if (recon != ORC_FIRST_ORDER) {
                            round_trip(&x->eos, ul);
                            round_trip(&x->eos, ur);
                        }
                        continue;
                    }
                    /* the stencil: cells t - pad .. t + pad - 1 along the axis, primitive */
                    St Ws[6];
                    for (int s = 0; s < 2 * pad; ++s) {
                        int cc[3] = {i, j, k};
                        cc[axis] = t - pad + s;
                        St Uc;
                        outside_state(x, U, kind, ut, cc[0], cc[1], cc[2], Uc);
                        c2p(&x->eos, Uc, Ws[s], NULL);
                    }
                    St wl, wr;
                    for (int q = 0; q < NV; ++q) {
                        if (recon == ORC_MUSCL) {
                            if (planar && q == 4) {
                                wl[q] = wr[q] = 0.0;
                                continue;
                            }
                            const double c0 = Ws[0][q], c1 = Ws[1][q], c2 = Ws[2][q], c3 = Ws[3][q];
                            const double b = c2 - c1;
                            wl[q] = c1 + 0.5 * apply_limiter(c->limiter, c1 - c0, b);
                            wr[q] = c2 - 0.5 * apply_limiter(c->limiter, c3 - c2, b);
                        } else if (recon == ORC_WENO3) {
                            wl[q] = weno3z(Ws[0][q], Ws[1][q], Ws[2][q], c->weno_eps);
                            wr[q] = weno3z(Ws[3][q], Ws[2][q], Ws[1][q], c->weno_eps);
                        } else {
                            wl[q] = weno5z(Ws[0][q], Ws[1][q], Ws[2][q], Ws[3][q], Ws[4][q], c->weno_eps);
                            wr[q] = weno5z(Ws[5][q], Ws[4][q], Ws[3][q], Ws[2][q], Ws[1][q], c->weno_eps);
                        }
                    }
                    p2c(&x->eos, wl, ul);
                    p2c(&x->eos, wr, ur);
                }
    }
    return 0;
}

/* ---------------------------------------------------------------- MUSCL-Hancock predictor (Schemes.cpp:2135-2200, 2888-3060) */
static void euler_flux_axis3(const Eos* e, const double* U, int a, double* F) {
    St W;
    c2p(e, U, W, NULL);
    const double un = a == 0 ? W[1] : a == 1 ? W[2] : W[4], p = W[3];
    F[0] = U[0] * un;
    F[1] = U[1] * un + (a == 0 ? p : 0.0);
    F[2] = U[2] * un + (a == 1 ? p : 0.0);
    F[3] = (U[3] + p) * un;
    F[4] = U[4] * un + (a == 2 ? p : 0.0);
}
static void euler_flux_axis(const Eos* e, const double* U, int a, double* F) {
    St W;
    c2p(e, U, W, NULL);
    const double un = a == 0 ? W[1] : W[2], p = W[3];
    F[0] = U[0] * un;
    F[1] = U[1] * un + (a == 0 ? p : 0.0);
    F[2] = U[2] * un + (a == 1 ? p : 0.0);
    F[3] = (U[3] + p) * un;
    F[4] = U[4] * un;
}
static int admissible_state(const Eos* e, const double* U) {
    if (!(U[0] > kEosEps)) return 0;
    return 0.5 * (U[1] * U[1] + U[2] * U[2] + U[4] * U[4]) < U[0] * (U[3] - e->p_inf);
}

/* hancock_predict / hancock_predict_3d (two-pass form, which the reference's fused pass reproduces bit for bit) followed by
 * hancock_wall_ghosts: the states of every cell advanced by half a step with its own flux difference. */
static void hancock(const Ctx* x, double* UL, double* UR, double half_dt, const int wrap[3]) {
    const Faces F = faces_of(x);
    const int nx = x->nx, ny = x->ny, nz = x->nz;
    const double hx = half_dt / x->dx, hy = half_dt / x->dy, hz = half_dt / x->dz;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double* st[6] = {UR + NV * xface(x, i, j, k), UL + NV * xface(x, i + 1, j, k), UR + NV * yface(x, &F, i, j, k),
                                 UL + NV * yface(x, &F, i, j + 1, k), NULL, NULL};
                const int ns = x->three_d ? 6 : 4;
                if (x->three_d) {
                    st[4] = UR + NV * zface(x, &F, i, j, k);
                    st[5] = UL + NV * zface(x, &F, i, j, k + 1);
                }
                St fl[6], d;
                for (int s = 0; s < ns; ++s) {
                    if (x->three_d)
                        euler_flux_axis3(&x->eos, st[s], s / 2, fl[s]);
                    else
                        euler_flux_axis(&x->eos, st[s], s / 2, fl[s]);
                }
                for (int q = 0; q < NV; ++q) {
                    if (x->three_d)
                        d[q] = (hx * (fl[1][q] - fl[0][q]) + hy * (fl[3][q] - fl[2][q])) + hz * (fl[5][q] - fl[4][q]);
                    else
                        d[q] = hx * (fl[1][q] - fl[0][q]) + hy * (fl[3][q] - fl[2][q]);
                }
                for (int s = 0; s < ns; ++s) {
                    St nn;
                    for (int q = 0; q < NV; ++q) nn[q] = st[s][q] - d[q];
                    if (admissible_state(&x->eos, nn)) memcpy(st[s], nn, sizeof(St));
                }
            }
    /* the two copies of a periodic seam face hold the states of the cells on either side */
    if (wrap[0])
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) {
                memcpy(UL + NV * xface(x, 0, j, k), UL + NV * xface(x, nx, j, k), sizeof(St));
                memcpy(UR + NV * xface(x, nx, j, k), UR + NV * xface(x, 0, j, k), sizeof(St));
            }
    if (wrap[1])
        for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx; ++i) {
                memcpy(UL + NV * yface(x, &F, i, 0, k), UL + NV * yface(x, &F, i, ny, k), sizeof(St));
                memcpy(UR + NV * yface(x, &F, i, ny, k), UR + NV * yface(x, &F, i, 0, k), sizeof(St));
            }
    if (wrap[2] && x->three_d)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                memcpy(UL + NV * zface(x, &F, i, j, 0), UL + NV * zface(x, &F, i, j, nz), sizeof(St));
                memcpy(UR + NV * zface(x, &F, i, j, nz), UR + NV * zface(x, &F, i, j, 0), sizeof(St));
            }
    /* walls: the ghost of the predicted state of the cell next to them (hancock_wall_ghosts, Schemes.cpp:2958-2982) */
    for (int s = 0; s < (x->three_d ? 6 : 4); ++s) {
        const int bt = x->c->bc[s];
        if (!(bt == ORC_WALL || bt == ORC_NOSLIP || bt == ORC_MOVINGWALL)) continue;
        const int a = s / 2, hi = s & 1, na = n_axis(x, a);
        const int n0 = a == 0 ? ny : nx, n1 = a == 2 ? ny : nz;
        for (int b = 0; b < n1; ++b)
            for (int q = 0; q < n0; ++q) {
                int i, j, k;
                if (a == 0) { i = hi ? na : 0; j = q; k = b; }
                else if (a == 1) { i = q; j = hi ? na : 0; k = b; }
                else { i = q; j = b; k = hi ? na : 0; }
                const size_t f = face_of(x, &F, a, i, j, k);
                if (hi)
                    ghost_state(x, s, UL + NV * f, 0.0, UR + NV * f);
                else
                    ghost_state(x, s, UR + NV * f, 0.0, UL + NV * f);
            }
    }
}

/* ---------------------------------------------------------------- viscous fluxes, 3-D (Physics.cpp:484-830, Boundaries.cpp:569-702) */
static inline size_t pidx3(const Ctx* x, int ii, int jj, int kk) { return ((size_t)kk * (x->ny + 2) + jj) * (x->nx + 2) + ii; }

/* the zero-gradient copy with the momentum rules of one side (BoundaryManager::viscous_ghost_3d, Boundaries.cpp:258-275) */
static void viscous_ghost_3d(const Ctx* x, int side, const double* c, double* gh) {
    memcpy(gh, c, sizeof(St));
    const double uw[3] = {x->c->u_in, x->c->v_in, 0.0};
    const int d = side / 2;
    switch (x->c->bc[side]) {
    case ORC_NOSLIP:
        for (int q = 0; q < 3; ++q) gh[kMom[q]] = -c[kMom[q]];
        break;
    case ORC_WALL: gh[kMom[d]] = -c[kMom[d]]; break;
    case ORC_MOVINGWALL:
        for (int t = 0; t < 3; ++t) gh[kMom[t]] = (t == d) ? -c[kMom[t]] : 2.0 * c[0] * uw[t] - c[kMom[t]];
        if (x->c->boundary_order == 2) /* match_kinetic_energy (Boundaries.cpp:197-200) */
            gh[3] = c[3] + 0.5 * (gh[1] * gh[1] + gh[2] * gh[2] + gh[4] * gh[4] - c[1] * c[1] - c[2] * c[2] - c[4] * c[4]) / c[0];
        break;
    default: break;
    }
}

/* BoundaryManager::padded_3d (Boundaries.cpp:621-700) then fix_padded_corners (Boundaries.cpp:509-548) */
static void padded_3d(const Ctx* x, const double* U, double* P) {
    const int nx = x->nx, ny = x->ny, nz = x->nz;
    for (int kk = 0; kk < nz + 2; ++kk) {
        const int k = kk - 1 < 0 ? 0 : (kk - 1 > nz - 1 ? nz - 1 : kk - 1);
        for (int jj = 0; jj < ny + 2; ++jj) {
            const int j = jj - 1 < 0 ? 0 : (jj - 1 > ny - 1 ? ny - 1 : jj - 1);
            for (int ii = 0; ii < nx + 2; ++ii) {
                const int i = ii - 1 < 0 ? 0 : (ii - 1 > nx - 1 ? nx - 1 : ii - 1);
                memcpy(P + NV * pidx3(x, ii, jj, kk), U + NV * cell(x, i, j, k), sizeof(St));
            }
        }
    }
    const int order[6] = {2, 3, 0, 1, 4, 5}; /* bottom, top, left, right, front, back */
    for (int o = 0; o < 6; ++o) {
        const int side = order[o], bc = x->c->bc[side];
        if (bc != ORC_NOSLIP && bc != ORC_WALL && bc != ORC_MOVINGWALL && bc != ORC_PERIODIC) continue;
        const int d = side / 2, hi = side & 1;
        const int n_d = d == 0 ? nx : (d == 1 ? ny : nz);
        const int g = hi ? n_d + 1 : 0, in = hi ? n_d - 1 : 0, op = hi ? 0 : n_d - 1;
        const int na = d == 0 ? ny : nx, nb = d == 2 ? ny : nz;
        for (int b = 0; b < nb; ++b)
            for (int a = 0; a < na; ++a) {
                int i, j, k, ii, jj, kk, io, jo, ko;
                if (d == 0) { i = in; j = a; k = b; ii = g; jj = j + 1; kk = k + 1; io = op; jo = j; ko = k; }
                else if (d == 1) { i = a; j = in; k = b; ii = i + 1; jj = g; kk = k + 1; io = i; jo = op; ko = k; }
                else { i = a; j = b; k = in; ii = i + 1; jj = j + 1; kk = g; io = i; jo = j; ko = op; }
                double* gh = P + NV * pidx3(x, ii, jj, kk);
                if (bc == ORC_PERIODIC)
                    memcpy(gh, U + NV * cell(x, io, jo, ko), sizeof(St));
                else
                    viscous_ghost_3d(x, side, U + NV * cell(x, i, j, k), gh);
            }
    }
    if (x->c->boundary_order != 2) return;
    const int n3[3] = {nx, ny, nz};
    for (int kk = 0; kk <= nz + 1; ++kk)
        for (int jj = 0; jj <= ny + 1; ++jj)
            for (int ii = 0; ii <= nx + 1; ++ii) {
                const int p[3] = {ii, jj, kk};
                int ng = 0, ga[2] = {-1, -1};
                for (int a = 0; a < 3; ++a)
                    if (p[a] == 0 || p[a] == n3[a] + 1) {
                        if (ng < 2) ga[ng] = a;
                        ++ng;
                    }
                if (ng != 2) continue;
                const int d = ga[0];
                const int hi = p[d] != 0;
                int q[3] = {p[0], p[1], p[2]};
                q[d] = hi ? n3[d] : 1;
                St cst, g;
                memcpy(cst, P + NV * pidx3(x, q[0], q[1], q[2]), sizeof(St));
                const int side = 2 * d + (hi ? 1 : 0);
                if (x->c->bc[side] == ORC_PERIODIC) {
                    q[d] = hi ? 1 : n3[d];
                    memcpy(g, P + NV * pidx3(x, q[0], q[1], q[2]), sizeof(St));
                } else {
                    viscous_ghost_3d(x, side, cst, g);
                }
                memcpy(P + NV * pidx3(x, ii, jj, kk), g, sizeof(St));
            }
}

/* NavierStokes::viscous_residual_3d, accumulated into R; returns the viscous speed bound */
static double viscous_3d(const Ctx* x, const double* U, double* R) {
    const int nx = x->nx, ny = x->ny, nz = x->nz;
    const size_t n = (size_t)nx * ny * nz, np = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    const double h[3] = {x->dx, x->dy, x->dz};
    const double gamma = x->eos.gamma, mu = x->c->mu;
    const double k_cond = mu * gamma / (x->c->pr * (gamma - 1.0)); /* TransportLaw (Core.hpp:194-197) */
    double* P = malloc(sizeof(St) * np);
    double* Wp = malloc(sizeof(St) * np);
    double* vel = malloc(sizeof(double) * 13 * n);
    padded_3d(x, U, P);
    for (size_t c = 0; c < np; ++c) c2p(&x->eos, P + NV * c, Wp + NV * c, NULL);
    double* sT = vel + 3 * n;
    double* G = vel + 4 * n; /* G[(3a + b) n + c] */
#define WPAD(ii, jj, kk) (Wp + NV * pidx3(x, (ii), (jj), (kk)))
#define UPAD(ii, jj, kk) (P + NV * pidx3(x, (ii), (jj), (kk)))
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t cc = cell(x, i, j, k);
                const double* w = WPAD(i + 1, j + 1, k + 1);
                const double rho = w[0];
                sT[cc] = w[3] / rho;
                const double* nb[3][2] = {{UPAD(i, j + 1, k + 1), UPAD(i + 2, j + 1, k + 1)},
                                          {UPAD(i + 1, j, k + 1), UPAD(i + 1, j + 2, k + 1)},
                                          {UPAD(i + 1, j + 1, k), UPAD(i + 1, j + 1, k + 2)}};
                double grad[3][5];
                for (int b = 0; b < 3; ++b)
                    for (int q = 0; q < 5; ++q)
                        if (q != 3) grad[b][q] = (nb[b][1][q] - nb[b][0][q]) / (2.0 * h[b]);
                for (int a = 0; a < 3; ++a) {
                    const double ua = w[kMom[a]];
                    vel[a * n + cc] = ua;
                    for (int b = 0; b < 3; ++b) G[(3 * a + b) * n + cc] = (grad[b][kMom[a]] - ua * grad[b][0]) / rho;
                }
            }
    const int periodic[3] = {x->c->bc[0] == ORC_PERIODIC && x->c->bc[1] == ORC_PERIODIC, x->c->bc[2] == ORC_PERIODIC && x->c->bc[3] == ORC_PERIODIC,
                             x->c->bc[4] == ORC_PERIODIC && x->c->bc[5] == ORC_PERIODIC};
    const int bface2 = x->c->boundary_order == 2;
    const double area[3] = {x->dy * x->dz, x->dx * x->dz, x->dx * x->dy};
    const Faces F = faces_of(x);
    double* FV = malloc(sizeof(St) * F.n);
    for (int d = 0; d < 3; ++d) {
        const int n_d = d == 0 ? nx : (d == 1 ? ny : nz);
        const int ni = nx + (d == 0), nj = ny + (d == 1), nk = nz + (d == 2);
        for (int k = 0; k < nk; ++k)
            for (int j = 0; j < nj; ++j)
                for (int i = 0; i < ni; ++i) {
                    const int idx[3] = {i, j, k};
                    const int t = idx[d];
                    const int lo = t == 0, hi = t == n_d;
                    int c3[3] = {i, j, k};
                    c3[d] = lo ? 0 : t - 1;
                    const size_t cL = cell(x, c3[0], c3[1], c3[2]);
                    c3[d] = hi ? n_d - 1 : t;
                    const size_t cR = cell(x, c3[0], c3[1], c3[2]);
                    double vL[3], vR[3], TL, TR;
                    if (lo) {
                        int p3[3] = {i + 1, j + 1, k + 1};
                        p3[d] = 0;
                        const double* g = WPAD(p3[0], p3[1], p3[2]);
                        for (int a = 0; a < 3; ++a) vL[a] = g[kMom[a]];
                        TL = g[3] / g[0];
                    } else {
                        for (int a = 0; a < 3; ++a) vL[a] = vel[a * n + cL];
                        TL = sT[cL];
                    }
                    if (hi) {
                        int p3[3] = {i + 1, j + 1, k + 1};
                        p3[d] = n_d + 1;
                        const double* g = WPAD(p3[0], p3[1], p3[2]);
                        for (int a = 0; a < 3; ++a) vR[a] = g[kMom[a]];
                        TR = g[3] / g[0];
                    } else {
                        for (int a = 0; a < 3; ++a) vR[a] = vel[a * n + cR];
                        TR = sT[cR];
                    }
                    c3[d] = n_d - 1;
                    const size_t xL = (lo && periodic[d]) ? cell(x, c3[0], c3[1], c3[2]) : cL;
                    c3[d] = 0;
                    const size_t xR = (hi && periodic[d]) ? cell(x, c3[0], c3[1], c3[2]) : cR;
                    const int phys = bface2 && !periodic[d] && (lo || hi);
                    double Gn[3], vf[3];
                    for (int a = 0; a < 3; ++a) {
                        Gn[a] = (vR[a] - vL[a]) / h[d];
                        vf[a] = 0.5 * (vL[a] + vR[a]);
                    }
                    const double dT = (TR - TL) / h[d];
                    double Gc[3][3] = {{0}};
                    int pairs[4][2];
                    if (d == 0) { int pp[4][2] = {{0, 1}, {1, 1}, {2, 2}, {0, 2}}; memcpy(pairs, pp, sizeof pp); }
                    else if (d == 1) { int pp[4][2] = {{0, 0}, {1, 0}, {2, 2}, {1, 2}}; memcpy(pairs, pp, sizeof pp); }
                    else { int pp[4][2] = {{0, 0}, {1, 1}, {2, 0}, {2, 1}}; memcpy(pairs, pp, sizeof pp); }
                    for (int w = 0; w < 4; ++w) {
                        const int a = pairs[w][0], b = pairs[w][1];
                        double val;
                        if (phys) {
                            int pg[3] = {i + 1, j + 1, k + 1}, pc[3] = {i + 1, j + 1, k + 1};
                            pg[d] = lo ? 0 : n_d + 1;
                            pc[d] = lo ? 1 : n_d;
                            double fc[2];
                            for (int s = 0; s < 2; ++s) {
                                const int off = s == 0 ? 1 : -1;
                                int g3[3] = {pg[0], pg[1], pg[2]}, q3[3] = {pc[0], pc[1], pc[2]};
                                g3[b] += off;
                                q3[b] += off;
                                fc[s] = 0.5 * (WPAD(g3[0], g3[1], g3[2])[kMom[a]] + WPAD(q3[0], q3[1], q3[2])[kMom[a]]);
                            }
                            val = (fc[0] - fc[1]) / (2.0 * h[b]);
                        } else {
                            val = 0.5 * (G[(3 * a + b) * n + xL] + G[(3 * a + b) * n + xR]);
                        }
                        Gc[a][b] = val;
                    }
                    double tau[3];
                    for (int a = 0; a < 3; ++a) {
                        if (a == d) {
                            double others = 0.0;
                            for (int o = 0; o < 3; ++o)
                                if (o != d) others += Gc[o][o];
                            tau[a] = mu * ((4.0 / 3.0) * Gn[d] - (2.0 / 3.0) * others);
                        } else {
                            tau[a] = mu * (Gn[a] + Gc[d][a]);
                        }
                    }
                    const double q_d = -k_cond * dT;
                    double* out = FV + NV * face_of(x, &F, d, i, j, k);
                    out[0] = 0.0;
                    out[1] = tau[0] * area[d];
                    out[2] = tau[1] * area[d];
                    out[3] = (vf[0] * tau[0] + vf[1] * tau[1] + vf[2] * tau[2] - q_d) * area[d];
                    out[4] = tau[2] * area[d];
                }
    }
    const double inv_vol = 1.0 / (x->dx * x->dy * x->dz);
    const double inv_h2 = 1.0 / (x->dx * x->dx) + 1.0 / (x->dy * x->dy) + 1.0 / (x->dz * x->dz);
    const double L = 2.0 / (1.0 / (x->c->Lx / nx) + 1.0 / (x->c->Ly / ny) + 1.0 / (x->c->Lz / nz));
    double s_max = 0.0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double* fl = FV + NV * xface(x, i, j, k);
                const double* fr = FV + NV * xface(x, i + 1, j, k);
                const double* fb = FV + NV * yface(x, &F, i, j, k);
                const double* ft = FV + NV * yface(x, &F, i, j + 1, k);
                const double* ff = FV + NV * zface(x, &F, i, j, k);
                const double* fk = FV + NV * zface(x, &F, i, j, k + 1);
                double* r = R + NV * cell(x, i, j, k);
                for (int q = 0; q < NV; ++q) r[q] += (((0.0 + (fr[q] - fl[q])) + (ft[q] - fb[q])) + (fk[q] - ff[q])) * inv_vol;
                const double* w = WPAD(i + 1, j + 1, k + 1);
                const double rho = w[0];
                const double nu_eff = dmax((4.0 / 3.0) * (mu / rho), (k_cond * (gamma - 1.0)) / rho) + 1e-12;
                const double vmax = dmax(dmax(fabs(w[1]), fabs(w[2])), fabs(w[4]));
                const double s = vmax + sound_speed(&x->eos, w[3], rho) + 2.0 * L * inv_h2 * nu_eff;
                s_max = dmax(s_max, s);
            }
#undef WPAD
#undef UPAD
    free(FV);
    free(vel);
    free(Wp);
    free(P);
    return s_max;
}

/* ---------------------------------------------------------------- residual */
int orc_residual(const orc_config* c, const double* U, double* R, double predictor_half_dt, double* smax) {
    Ctx x;
    ctx_init(&x, c);
    if (c->viscous && !x.three_d) return -4; /* the 2-D viscous sweep is not restated */
    if (predictor_half_dt > 0.0 && c->recon != ORC_MUSCL) return -5;
    for (int a = 0; a < (x.three_d ? 3 : 2); ++a)
        if ((c->bc[2 * a] == ORC_PERIODIC) != (c->bc[2 * a + 1] == ORC_PERIODIC)) return -6;
    const Faces F = faces_of(&x);
    double* UL = malloc(sizeof(St) * F.n);
    double* UR = malloc(sizeof(St) * F.n);
    double* FF = malloc(sizeof(St) * F.n);
    double ut[6];
    for (int s = 0; s < 6; ++s) ut[s] = u_target_of(&x, U, s);
    int rc = face_states(&x, U, ut, UL, UR);
    if (rc) goto done;
    if (predictor_half_dt > 0.0) {
        int kind[6], wrap[3];
        halo_kinds(&x, 2, kind);
        for (int a = 0; a < 3; ++a) wrap[a] = kind[2 * a] == 1 && kind[2 * a + 1] == 1;
        hancock(&x, UL, UR, predictor_half_dt, wrap);
    }
    double S = 0.0;
    for (size_t f = 0; f < F.n; ++f) {
        const int axis = f < F.nxf ? 0 : (f < F.nxf + F.nyf ? 1 : 2);
        const double s = face_flux(&x.rs, UL + NV * f, UR + NV * f, axis, FF + NV * f);
        if (s > S) S = s;
    }
    const int nx = x.nx, ny = x.ny, nz = x.nz;
    if (!x.three_d) {
        const double inv_area = 1.0 / (x.dx * x.dy), dxl = x.dx, dyl = x.dy;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double* fl = FF + NV * xface(&x, i, j, 0);
                const double* fr = FF + NV * xface(&x, i + 1, j, 0);
                const double* fb = FF + NV * yface(&x, &F, i, j, 0);
                const double* ft = FF + NV * yface(&x, &F, i, j + 1, 0);
                double* r = R + NV * cell(&x, i, j, 0);
                for (int q = 0; q < NV; ++q) r[q] = ((0.0 - (fr[q] * dyl - fl[q] * dyl)) - (ft[q] * dxl - fb[q] * dxl)) * inv_area;
            }
    } else {
        const double Ax = x.dy * x.dz, Ay = x.dx * x.dz, Az = x.dx * x.dy, inv_vol = 1.0 / (x.dx * x.dy * x.dz);
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double* fl = FF + NV * xface(&x, i, j, k);
                    const double* fr = FF + NV * xface(&x, i + 1, j, k);
                    const double* fb = FF + NV * yface(&x, &F, i, j, k);
                    const double* ft = FF + NV * yface(&x, &F, i, j + 1, k);
                    const double* ff = FF + NV * zface(&x, &F, i, j, k);
                    const double* fk = FF + NV * zface(&x, &F, i, j, k + 1);
                    double* r = R + NV * cell(&x, i, j, k);
                    for (int q = 0; q < NV; ++q)
                        r[q] = (((0.0 - (fr[q] * Ax - fl[q] * Ax)) - (ft[q] * Ay - fb[q] * Ay)) - (fk[q] * Az - ff[q] * Az)) * inv_vol;
                }
    }
    if (c->viscous) {
        const double sv = viscous_3d(&x, U, R);
        S = dmax(S, sv);
    }
    *smax = S;
done:
    free(UL);
    free(UR);
    free(FF);
    return rc;
}

double orc_dt_length(const orc_config* c) {
    const double dx = c->Lx / c->nx, dy = c->Ly / c->ny;
    if (c->nz > 1) return 2.0 / (1.0 / dx + 1.0 / dy + 1.0 / (c->Lz / c->nz));
    return dmin(dx, dy);
}

/* ---------------------------------------------------------------- time schemes (TimeScheme.cpp:110-319) */
int orc_step(const orc_config* c, double* U, double t, double t_end, double* lagged, double* dt_out, double* smax_out) {
    const size_t n = (size_t)c->nx * c->ny * c->nz * NV;
    const double L = orc_dt_length(c);
    double* R = malloc(sizeof(double) * n);
    double* tmp = malloc(sizeof(double) * n);
    int rc = 0;
    double s1 = 0.0, s2 = 0.0, s3 = 0.0, dt = 0.0;
#define CLAMP_DT(s)                                   \
    dt = c->cfl * L / ((s) + kDtEps);                 \
    dt = dmin(dt, t_end - t);                         \
    if (c->dt_max > 0.0) dt = dmin(dt, c->dt_max);
    if (c->time_scheme == ORC_HANCOCK) {
        if (!(*lagged > 0.0)) {
            if ((rc = orc_residual(c, U, R, 0.0, lagged))) goto out;
        }
        CLAMP_DT(*lagged);
        if ((rc = orc_residual(c, U, R, 0.5 * dt, &s1))) goto out;
        for (size_t e = 0; e < n; ++e) U[e] = U[e] + dt * R[e];
        *lagged = s1;
        *smax_out = s1;
    } else {
        if ((rc = orc_residual(c, U, R, 0.0, &s1))) goto out;
        CLAMP_DT(s1);
        if (c->time_scheme == ORC_EULER) {
            for (size_t e = 0; e < n; ++e) U[e] = U[e] + dt * R[e];
            *smax_out = s1;
        } else {
            for (size_t e = 0; e < n; ++e) tmp[e] = U[e] + dt * R[e];
            if ((rc = orc_residual(c, tmp, R, 0.0, &s2))) goto out;
            if (c->time_scheme == ORC_SSPRK2) {
                for (size_t e = 0; e < n; ++e) U[e] = 0.5 * U[e] + 0.5 * (tmp[e] + dt * R[e]);
                *smax_out = dmax(s1, s2);
            } else {
                for (size_t e = 0; e < n; ++e) tmp[e] = 0.75 * U[e] + 0.25 * (tmp[e] + dt * R[e]);
                if ((rc = orc_residual(c, tmp, R, 0.0, &s3))) goto out;
                for (size_t e = 0; e < n; ++e) U[e] = (1.0 / 3.0) * U[e] + (2.0 / 3.0) * (tmp[e] + dt * R[e]);
                *smax_out = dmax(s1, dmax(s2, s3));
            }
        }
    }
    *dt_out = dt;
#undef CLAMP_DT
out:
    free(R);
    free(tmp);
    return rc;
}

/* ---------------------------------------------------------------- Riemann fingerprint (cpp/apps/bench_riemann.cpp) */
typedef struct {
    uint64_t s;
} Lcg;
static double lcg_next(Lcg* g) {
    g->s = g->s * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(g->s >> 11) * (1.0 / 9007199254740992.0);
}
static uint64_t bits_of(double x) {
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
}

void orc_riemann_pool(int eos_kind, double* UL, double* UR, int* axis) {
    const int pool = 1 << 16;
    Eos eos = {eos_kind == 0 ? ORC_IDEAL : ORC_STIFFENED, eos_kind == 0 ? 1.4 : 4.4, eos_kind == 0 ? 0.0 : 6.0e8};
    Lcg rng = {88172645463325252ull};
    for (int k = 0; k < pool; ++k) {
        const int strong = lcg_next(&rng) < 0.1;
        const double p0 = eos_kind == 0 ? 1.0 : 1.0e8;
        St a;
        a[0] = 1.0 + 0.2 * lcg_next(&rng);
        a[1] = 2.0 * lcg_next(&rng) - 1.0;
        a[2] = 2.0 * lcg_next(&rng) - 1.0;
        a[3] = p0 * (1.0 + 0.2 * lcg_next(&rng));
        a[4] = 2.0 * lcg_next(&rng) - 1.0;
        St b;
        memcpy(b, a, sizeof(St));
        const double jump = strong ? 4.0 : 0.02;
        b[0] *= 1.0 + jump * lcg_next(&rng);
        b[1] += jump * (lcg_next(&rng) - 0.5);
        b[2] += jump * (lcg_next(&rng) - 0.5);
        b[3] *= 1.0 + jump * lcg_next(&rng);
        b[4] += 0.1 * jump * (lcg_next(&rng) - 0.5);
        p2c(&eos, a, UL + NV * k);
        p2c(&eos, b, UR + NV * k);
        axis[k] = (int)(lcg_next(&rng) * 3.0) % 3;
    }
    int k = 0;
    const double p0 = eos_kind == 0 ? 1.0 : 1.0e8;
#define PUT(l, r, ax)                              \
    do {                                           \
        memcpy(UL + NV * k, (l), sizeof(St));      \
        memcpy(UR + NV * k, (r), sizeof(St));      \
        axis[k] = (ax);                            \
        ++k;                                       \
    } while (0)
    for (int ax = 0; ax < 3; ++ax) {
        St a, b, w1, w2;
        const St wa = {1.0, 0.3, -0.2, p0, 0.1};
        p2c(&eos, wa, a);
        PUT(a, a, ax);
        const St wb = {1.0, -0.3, -0.2, p0, 0.1};
        p2c(&eos, wa, a);
        p2c(&eos, wb, b);
        PUT(a, b, ax);
        const St wc = {1.0, 0.0, 0.0, p0, 0.0}, wd = {0.125, -0.0, 0.0, 0.1 * p0, -0.0};
        p2c(&eos, wc, w1);
        p2c(&eos, wd, w2);
        PUT(w1, w2, ax);
        const St we = {1.0, 0.0, 0.0, 2.0 * p0, 0.0};
        p2c(&eos, wc, w1);
        p2c(&eos, we, w2);
        PUT(w1, w2, ax);
        const St r0 = {1e-20, 0.0, 0.0, 1e-20, 0.0}, r1 = {1.0, 0.0, 0.0, p0, 0.0};
        PUT(r0, r1, ax);
        const St r2 = {1.0, 5.0, 0.0, 0.1, 0.0};
        PUT(r2, r2, ax);
        const St r3 = {-1.0, 1.0, 0.0, 1.0, 0.0};
        PUT(r3, r1, ax);
        for (int ulp = -2; ulp <= 2; ++ulp) {
            const double cs = sqrt(eos.gamma * (p0 + (eos_kind == 0 ? 0.0 : eos.p_inf)) / 1.0);
            double u = cs;
            for (int q = 0; q < abs(ulp); ++q) u = nextafter(u, ulp < 0 ? 0.0 : 1e300);
            St W = {1.0, 0.0, 0.0, p0, 0.0};
            W[ax == 0 ? 1 : (ax == 1 ? 2 : 4)] = u;
            St Wr;
            memcpy(Wr, W, sizeof(St));
            Wr[3] *= 1.0 + 1e-3;
            p2c(&eos, W, w1);
            p2c(&eos, Wr, w2);
            PUT(w1, w2, ax);
            PUT(w2, w1, ax);
        }
    }
#undef PUT
}

unsigned long long orc_riemann_hash(int eos_kind, int riemann) {
    const int pool = 1 << 16;
    double* UL = malloc(sizeof(St) * pool);
    double* UR = malloc(sizeof(St) * pool);
    int* axis = malloc(sizeof(int) * pool);
    orc_riemann_pool(eos_kind, UL, UR, axis);
    Riemann rs = {{eos_kind == 0 ? ORC_IDEAL : ORC_STIFFENED, eos_kind == 0 ? 1.4 : 4.4, eos_kind == 0 ? 0.0 : 6.0e8}, riemann, 0.0};
    uint64_t h = 1469598103934665603ull;
    for (int k = 0; k < pool; ++k) {
        St F;
        const double sm = face_flux(&rs, UL + NV * k, UR + NV * k, axis[k], F);
        for (int q = 0; q < NV; ++q) h = (h ^ bits_of(F[q])) * 1099511628211ull;
        h = (h ^ bits_of(sm)) * 1099511628211ull;
    }
    free(UL);
    free(UR);
    free(axis);
    return (unsigned long long)h;
}

double orc_face_flux(const orc_config* c, const double* UL, const double* UR, int axis, double* F) {
    Riemann rs = {{c->eos, c->gamma, c->p_inf}, c->riemann, c->shock_blend};
    return face_flux(&rs, UL, UR, axis, F);
}
