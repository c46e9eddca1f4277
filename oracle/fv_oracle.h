/* CPU restatement of the reference's uniform-grid finite-volume right-hand side and time step (Fenice,
 * edotaglialatela/fenice). TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it, as the checker; the product never links or calls it.
 *
 * Every function restates the reference's arithmetic in the reference's operation order (the reference is built
 * with -ffp-contract=off and so is this file), so its results are the reference's bits. It is pinned against the
 * reference itself: tests/test_oracle_vs_ref.py compares it with the reference compiled from its own sources
 * (oracle/_ref, built by oracle/ref/Makefile) and with the golden fixtures under tests/golden/, which were written
 * by the reference (tests/golden/make_golden.py), and the Riemann solvers reproduce the reference's
 * bench_riemann fingerprint hashes.
 *
 * Layout: the reference's own, an array of cells of 5 doubles [rho, rho u, rho v, rho E, rho w], cell
 * (k*ny + j)*nx + i. */
#ifndef FV_ORACLE_H
#define FV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_IDEAL = 0, ORC_STIFFENED = 1 };
enum { ORC_HLLC = 0, ORC_LOWMACH = 1 };
enum { ORC_FIRST_ORDER = 0, ORC_MUSCL = 1, ORC_WENO3 = 2, ORC_WENO5 = 3 };
enum { ORC_MINMOD = 0, ORC_VANLEER = 1, ORC_MC = 2, ORC_KOREN = 3 };
/* boundary types, in the order of the reference's BCType (cpp/include/fv/Boundaries.hpp:15) */
enum { ORC_WALL = 0, ORC_NOSLIP, ORC_MOVINGWALL, ORC_VELINLET, ORC_MASSFLOWINLET, ORC_OUTLET, ORC_TRANSMISSIVE, ORC_PERIODIC,
       ORC_NONREFLECTING };
enum { ORC_EULER = 0, ORC_SSPRK2 = 1, ORC_SSPRK3 = 2, ORC_HANCOCK = 3 };

typedef struct {
    int nx, ny, nz;
    double Lx, Ly, Lz;
    int eos;
    double gamma, p_inf;
    int bc[6]; /* left, right, bottom, top, front, back */
    double u_in, v_in, rho_in, p_out;
    int riemann;
    double shock_blend;
    int recon, limiter;
    double weno_eps;
    int boundary_order;
    int time_scheme;
    double cfl, dt_max;
    int viscous;
    double mu, pr;
} orc_config;

/* Residual R(U) of the whole mesh (reference Simulation::assemble / assemble_3d, cpp/src/Simulation.cpp:811-1323), with
 * the MUSCL-Hancock predictor of half a step when predictor_half_dt > 0. Returns 0 and the wave speed in *smax, or a
 * negative code for a configuration the restatement does not cover. */
int orc_residual(const orc_config* c, const double* U, double* R, double predictor_half_dt, double* smax);

/* One step of the time scheme (reference TimeScheme::step, cpp/src/TimeScheme.cpp:110-319) on U in place, clamped to
 * t_end; *lagged is the MUSCL-Hancock wave speed of the previous step (0: none yet), updated. */
int orc_step(const orc_config* c, double* U, double t, double t_end, double* lagged, double* dt_out, double* smax_out);

/* The CFL length of the mesh (reference Simulation::setup, cpp/src/Simulation.cpp:225-227). */
double orc_dt_length(const orc_config* c);

/* The fingerprint of the reference's bench_riemann over one pass of its 65536 state pairs (cpp/apps/bench_riemann.cpp):
 * eos_kind 0 ideal (gamma 1.4), 1 stiffened (4.4, 6e8); riemann ORC_HLLC / ORC_LOWMACH; no shock blend. */
unsigned long long orc_riemann_hash(int eos_kind, int riemann);
/* The same state pairs (UL, UR: 65536 x 5 doubles, axis: 65536 ints), for a device solver to be hashed the same way. */
void orc_riemann_pool(int eos_kind, double* UL, double* UR, int* axis);
/* One face flux of the restated solver (F: 5 doubles), smax returned. */
double orc_face_flux(const orc_config* c, const double* UL, const double* UR, int axis, double* F);

#ifdef __cplusplus
}
#endif
#endif
