/* fenice_gpu.h: the C ABI of the B200 finite-volume path (libfenice_gpu.so).
 *
 * The reference (Fenice, C++17) has no C ABI: its hot path sits behind two C++ seams, which these entry points
 * replace one for one:
 *   - the residual seam  `using ResidualFn = std::function<double(const Field& U, Field& R)>`
 *     (cpp/include/fv/TimeScheme.hpp:14), evaluated by Simulation::residual (cpp/src/Simulation.cpp:1351-1354) with the
 *     scheme's stage_time / predictor_half_dt (cpp/include/fv/TimeScheme.hpp:88-92)           -> fvg_residual
 *   - the integrator seam `StepResult TimeScheme::step(Field& U, const ResidualFn&, double min_delta, double t,
 *     double t_max, double dt_max)` (cpp/include/fv/TimeScheme.hpp:48), driven by the serial time loop
 *     (cpp/src/SimulationRun.cpp:161-191, 441-464)                                             -> fvg_step, fvg_run
 * and the objects behind them are configured by one plain struct, the hot-path subset of the reference's SimParams
 * (cpp/include/fv/Params.hpp:57-147) that Simulation::setup turns into EOS, BoundaryManager, RiemannSolver,
 * MusclReconstruction, NavierStokes and TimeScheme (cpp/src/Simulation.cpp:188-360)              -> fvg_config, fvg_create.
 *
 * Conventions: plain pointers and sizes, no C++ types; every call returns an int status (FVG_OK = 0) and never throws;
 * fvg_last_error gives the message of the last failure of a handle. States cross the ABI in the reference's own layout:
 * an array of cells of 5 doubles [rho, rho u, rho v, rho E, rho w], cell (k*ny + j)*nx + i (cpp/include/fv/Core.hpp:20-24,114).
 * One host thread per handle; each handle owns a CUDA stream.
 */
#ifndef FENICE_GPU_H
#define FENICE_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FVG_ABI_VERSION 9

/* status codes */
enum {
    FVG_OK = 0,
    FVG_ERR_CONFIG = 1,      /* invalid or unsupported configuration */
    FVG_ERR_ARGUMENT = 2,    /* bad pointer or size */
    FVG_ERR_CUDA = 3,        /* a CUDA call failed (no device, out of memory, launch failure) */
    FVG_ERR_DIVERGED = 4,    /* non-finite wave speed or time step, or t no longer advances (check_progress) */
    FVG_ERR_STATE = 5,       /* the state is not valid for the mesh (e.g. rho w != 0 on a 2-D mesh) */
    FVG_ERR_BOUNDARY = 6     /* a time-dependent boundary value was not finite, or rho_in or p_out not positive, at a
                                stage time (Simulation::update_boundary_values, cpp/src/Simulation.cpp:170-185) */
};

/* enumerations, in the reference's order */
enum { FVG_EOS_IDEAL = 0, FVG_EOS_STIFFENED = 1 };                                  /* EOS::Type */
enum { FVG_RIEMANN_HLLC = 0, FVG_RIEMANN_LOWMACH = 1 };                             /* RiemannType */
enum { FVG_RECON_NONE = 0, FVG_RECON_MUSCL = 1, FVG_RECON_WENO3 = 2, FVG_RECON_WENO5 = 3 };
enum { FVG_LIM_MINMOD = 0, FVG_LIM_VANLEER = 1, FVG_LIM_MC = 2, FVG_LIM_KOREN = 3 };  /* Limiter */
enum { FVG_BC_WALL = 0, FVG_BC_NOSLIP, FVG_BC_MOVINGWALL, FVG_BC_VELINLET, FVG_BC_MASSFLOWINLET, FVG_BC_OUTLET,
       FVG_BC_TRANSMISSIVE, FVG_BC_PERIODIC, FVG_BC_NONREFLECTING };                  /* BCType */
enum { FVG_TS_EULER = 0, FVG_TS_SSPRK2 = 1, FVG_TS_SSPRK3 = 2, FVG_TS_HANCOCK = 3 };  /* TimeSchemeType */
enum { FVG_PREC_FP64 = 0, FVG_PREC_MIXED = 1 };

/* The run configuration: the reference's hot-path parameters (their case-file keys in brackets). */
typedef struct fvg_config {
    int nx, ny, nz;              /* [mesh] nx, ny, nz (nz = 1: a 2-D mesh) */
    double Lx, Ly, Lz;           /* [mesh] Lx, Ly, Lz */
    int eos_type;                /* [thermo] eos_type */
    double gamma, p_inf;         /* [thermo] gamma, p_inf */
    int bc[6];                   /* [boundaries] bc_xmin, bc_xmax, bc_ymin, bc_ymax, bc_zmin, bc_zmax */
    double u_in, v_in, rho_in, p_out; /* [boundaries] */
    int riemann;                 /* [numerics] riemann_solver */
    double shock_blend;          /* [numerics] shock_blend (default 0.2) */
    int reconstruction;          /* [numerics] reconstruction */
    int limiter;                 /* [numerics] muscl_limiter */
    double weno_epsilon;         /* [numerics] weno_epsilon */
    int boundary_order;          /* [numerics] boundary_order (default 2) */
    int time_scheme;             /* [numerics] time_scheme (resolved: no "auto") */
    double cfl;                  /* [numerics] cfl */
    double dt_max;               /* [run] dt_max (0: none) */
    int use_viscous;             /* [physics] use_viscous */
    double mu, pr;               /* [physics] mu, pr */
    int precision;               /* FVG_PREC_FP64: the reference's arithmetic, bit for bit; FVG_PREC_MIXED: FP32 stencil */
    int device;                  /* CUDA device ordinal */
    int use_ibm;                 /* [ibm] use_ibm: a static immersed body with the sharp ghost-cell wall (slip when inviscid) */
    int ibm_shape;               /* [ibm] ibm_shape: 0 Cylinder (a circle in 2-D, infinite along z in 3-D), 1 Sphere (3-D),
                                    2 a section (NACAxxxx / airfoil: ibm_section below; extruded along z in 3-D) */
    double ibm_radius, ibm_cx, ibm_cy, ibm_cz; /* [ibm] */
    int ibm_curvature;           /* [ibm] ibm_curvature (must be 0 on the device) */
    int use_bodyforce;           /* [physics] use_bodyforce: the constant body force (ConstantBodyForce, Physics.cpp:832-844) */
    double gx, gy, gz;           /* [physics] gx, gy, gz (gz is not used on a 2-D mesh) */
    double nrbc_sigma, nrbc_beta; /* [boundaries] the non-reflecting outlet's relaxation (0.28) and transverse weight (-1: local Mach) */
    int positivity_fallback;     /* [numerics] positivity_fallback: a stage that leaves a cell without density or pressure is
                                    repeated with first-order faces around it (WENO3-Z / WENO5-Z, FP64) */
    /* Case-file expressions, in the reference's expression grammar (TinyExpr with right-to-left ^; a whole number is
     * read with strtod). They may use x, y, z (cell centres), t, the parameters param_names / param_values (bound in
     * order, a later name replacing an earlier one, as the reference's Evaluator binds every numeric run parameter,
     * cpp/src/CaseFile.cpp:299-333) and then Lx, Ly, Lz, nx, ny, nz of the mesh. FP64 form only. */
    const char* source[5];       /* [source] source_rho, source_mx, source_my, source_E, source_mz (NULL: "0"): the source
                                    terms added to R after the viscous term and the body force (RhsSourceTerms,
                                    cpp/include/fv/Physics.hpp:21-47, cpp/src/Simulation.cpp:397-412); evaluated once at
                                    t = 0, or at every stage time when one of them reads t (source_unsteady). source_mz
                                    must be 0 on a 2-D mesh. */
    const char* boundary_expr[4];      /* u_in, v_in, rho_in, p_out as expressions of t (NULL: the constants above) */
    const double* boundary_table[4];   /* or as time tables ([boundaries] u_in_table ...): boundary_table_rows[k] rows of
                                          (t, value), linear between rows, constant outside (read_time_table /
                                          table_value, cpp/src/SimulationInternal.hpp:62-111) */
    int boundary_table_rows[4];
    const char* const* param_names;
    const double* param_values;
    int nparams;
    int flux_quadrature;         /* [numerics] flux_quadrature: 0 midpoint, 1 fourth (WENO3-Z / WENO5-Z of the conserved
                                    averages, point values at the face centres and the transverse flux correction,
                                    cpp/src/Schemes.cpp:1202-1350, 1954-2133; FP64, whole meshes without an immersed body) */
    /* [ibm] a prescribed motion of the body (Simulation::prescribed_pose, cpp/src/SimulationRun.cpp:193-214; a circle in
     * 2-D, a sphere in 3-D): constant velocity (ibm_vz: 3-D), angular velocity about z (2-D) or x and y (a sphere), and
     * the window of the rotation (0: always). The geometry follows the pose in steps of a quarter cell, the cells the
     * body leaves take the wall layer's state, the ghost states see the wall velocity (Physics.cpp:1128-1336, 1581-1637). */
    double ibm_vx, ibm_vy, ibm_vz;
    double ibm_omega, ibm_omega_x, ibm_omega_y;
    double ibm_omega_from, ibm_omega_until;
    /* [ibm] a body driven by the flow (Simulation::advance_body, cpp/src/SimulationRun.cpp:232-310): ibm_mass > 0 frees
     * its translation, ibm_inertia > 0 (about the pivot, ibm_cx, ibm_cy) its rotation; springs and dampers at the pivot;
     * the centre of mass off the pivot (2-D, ibm_cm_given). The loads are those of the first stage of each step; ibm_vx ..
     * ibm_omega_y are then the initial velocities. Runge-Kutta and Euler schemes only (as the reference). */
    double ibm_mass, ibm_inertia;
    double ibm_stiff_x, ibm_stiff_y, ibm_stiff_z, ibm_damp_x, ibm_damp_y, ibm_damp_z, ibm_stiff_theta, ibm_damp_theta;
    double ibm_cm_x, ibm_cm_y;
    int ibm_cm_given;
    /* [ibm] a section body (ibm_shape 2): the unit section's vertices (x, y pairs: leading edge at the origin, chord 1 along
     * x, as naca4 / load_airfoil give it, cpp/src/Geometry.cpp:40-141), placed by place_airfoil with its quarter chord at
     * (ibm_cx, ibm_cy), scaled to ibm_chord and turned by ibm_aoa degrees, nose up */
    const double* ibm_section;
    int ibm_section_points;
    double ibm_chord, ibm_aoa;
} fvg_config;

typedef struct fvg_run fvg_run;

/* A run on the device: validates the configuration, allocates the state and work arrays, and sets t = 0. */
int fvg_create(const fvg_config* cfg, fvg_run** out);
int fvg_destroy(fvg_run* run);
const char* fvg_last_error(const fvg_run* run);
/* A message for a failure of fvg_create (no handle exists then). */
const char* fvg_create_error(void);
int fvg_abi_version(void);

/* The state of the run (host arrays of ncells x 5 doubles, reference layout). */
int fvg_upload_state(fvg_run* run, const double* U, size_t ncells);
int fvg_download_state(fvg_run* run, double* U, size_t ncells);

/* Simulation::residual of the current state: R (host, ncells x 5, may be NULL) and the wave speed the residual returns;
 * predictor_half_dt > 0 applies the MUSCL-Hancock predictor of half a step (MUSCL only). */
int fvg_residual(fvg_run* run, double predictor_half_dt, double* R, size_t ncells, double* smax);

/* One step of the serial time loop from the run's time t toward t_end: TimeScheme::step, check_progress, t += dt.
 * dt and the step's wave speed are returned. */
int fvg_step(fvg_run* run, double t_end, double* dt, double* smax);

/* Steps until t >= t_end or `max_steps` steps were taken (max_steps <= 0: no limit), launched as CUDA graphs with the
 * clock kept on the device; *steps gets the number taken. */
int fvg_run_until(fvg_run* run, double t_end, int max_steps, int* steps);

/* TimeScheme::step(Field& U, ...) with U in host memory (cpp/include/fv/TimeScheme.hpp:48, the seam's caller owns U):
 * U_in (ncells x 5 doubles, reference layout) is uploaded, one step of the serial time loop taken toward t_end and the
 * new state written to U_out (which may be U_in); dt and the step's wave speed are returned. The result is the bits of
 * fvg_upload_state + fvg_step + fvg_download_state. For Runge-Kutta and Euler runs without an immersed body, mass-flow
 * inlet, positivity fallback or fourth-order quadrature, the copies overlap the computation: the state crosses the host
 * link in slabs along the slowest axis, the first stage starts on the slabs that have arrived and the last stage's slabs
 * are read back as they are finished (pinned host buffers are needed for the overlap). Other runs take the three calls
 * in turn. With the learned sensor, the gate is refreshed on every sens_every-th call that steps, counted from
 * fvg_set_sensor (fvg_step refreshes it on every call). */
int fvg_step_host(fvg_run* run, const double* U_in, double* U_out, size_t ncells, double t_end, double* dt, double* smax);

/* ---- Slab decomposition (one process, or one part, per GPU; SimulationRun.cpp:1011-1446 run_mpi and
 * MPIDecomposition.cpp:114-242 split the mesh into strips the same way and exchange halos and the wave speed).
 * Part `part` of `nparts` slabs of the mesh of cfg along its slowest axis (z on a 3-D mesh, y on a 2-D one): planes
 * first .. first + count - 1 (the first nsplit % nparts parts hold one plane more), with `depth` ghost planes beyond each
 * side that is an interface with a neighbouring part (a periodic axis joins the last part to the first). The mesh
 * spacing and step length are the whole mesh's, so a decomposed run gives the bits of the whole run. A part's state is
 * uploaded and downloaded with fvg_upload_state / fvg_download_state (its own cells, in the reference's order); it is
 * advanced step by step through fvg_part_phase (fvg_step, fvg_run_until, fvg_residual and the sensor are refused).
 * Refused configurations: an immersed body; fewer than depth (3 for WENO5, else 2) planes per part; a first-order run
 * split along a periodic axis. */
int fvg_create_part(const fvg_config* cfg, int nparts, int part, fvg_run** out);
/* axis: 1 (y) or 2 (z); the part's planes; ghost depth; whether the low / high side is an interface */
int fvg_part_info(const fvg_run* run, int* axis, int* first, int* count, int* depth, int* peer_lo, int* peer_hi);
/* the part's device buffers: the planes it sends to its low and high neighbours and receives from them (count doubles
 * each), and the all-reduce slots (2 doubles) */
int fvg_part_buffers(fvg_run* run, double** send_lo, double** send_hi, double** recv_lo, double** recv_hi, long long* count, double** reduce);
/* starts advancing toward t_end (max_steps > 0: at most that many steps), as fvg_run_until does */
int fvg_part_begin(fvg_run* run, double t_end, int max_steps);
/* Enqueues phase `phase` (0, 1, ...) of the current step on the run's stream. *comm says what the hosts do before the
 * next phase, on that stream: 0 the step is complete; 1 exchange: every part's send_lo goes to its low neighbour's
 * recv_hi and its send_hi to its high neighbour's recv_lo; 2 all-reduce (MAX, over all parts) the first *nreduce doubles
 * of the reduce slots. Every part takes the same phases in the same order. */
int fvg_part_phase(fvg_run* run, int phase, int* comm, int* nreduce);
/* reads the control block (synchronises the stream): whether the run continues, its steps, t, the last dt and wave
 * speed; FVG_ERR_DIVERGED as fvg_run_until */
int fvg_part_status(fvg_run* run, int* active, int* steps, double* t, double* dt, double* smax);

int fvg_get_time(const fvg_run* run, double* t);
int fvg_set_time(fvg_run* run, double t);
/* The time at which the next fvg_residual calls evaluate time-dependent source terms and boundary values
 * (TimeScheme::stage_time, cpp/include/fv/TimeScheme.hpp:88); NaN (the default): the run's time t, plus
 * predictor_half_dt for a MUSCL-Hancock residual. The time loop (fvg_step, fvg_run_until, parts) sets its own. */
int fvg_set_stage_time(fvg_run* run, double t);
/* Evaluates one case-file expression on the host (the C library's functions, the reference's values bit for bit) at n
 * points (x, y, z may be NULL: 0) and time t, with the names bound as in fvg_config. Returns FVG_OK, or FVG_ERR_CONFIG
 * with the reason in err (errlen bytes) for an expression the grammar refuses. */
int fvg_expr_eval(const char* expr, const char* const* names, const double* values, int nnames, const double* x, const double* y,
                  const double* z, double t, size_t n, double* out, char* err, size_t errlen);
/* The MUSCL-Hancock lagged wave speed (the reference's checkpoint key S; 0: the next step seeds it). */
int fvg_get_lagged_speed(const fvg_run* run, double* s);
int fvg_set_lagged_speed(fvg_run* run, double s);
/* The CFL length L in dt = cfl L / S (Simulation::setup, cpp/src/Simulation.cpp:225-227). */
int fvg_dt_length(const fvg_run* run, double* L);

/* Device access for callers that keep the state on the GPU (e.g. torch): the state planes (nvar planes of `plane`
 * doubles each, nvar = 4 on a 2-D mesh, 5 on a 3-D mesh) and the run's CUDA stream. */
int fvg_device_state(fvg_run* run, double** planes, long long* plane, int* nvar);
int fvg_stream(fvg_run* run, void** stream);
/* Wait for the run's stream. */
int fvg_synchronize(fvg_run* run);

/* Kernel timing: with `on`, fvg_run_until launches its steps one by one with CUDA events on the run's stream around
 * every launch of the stage kernel (reconstruction + Riemann + balance + update, or the MUSCL-Hancock kernel) and of the
 * viscous kernel; fvg_get_timing returns the summed device milliseconds and launch counts since timing was switched on. */
int fvg_set_timing(fvg_run* run, int on);
int fvg_get_timing(const fvg_run* run, double* stage_ms, long long* stage_launches, double* viscous_ms, long long* viscous_launches);

/* The immersed body's loads from a residual of the current state (Simulation::ibm_loads, cpp/src/SimulationRun.cpp:134-155,
 * and the monitor's coefficients, :94-103): loads[6] = {Fx, Fy, Mz, Cd, Cl, Cm}; F the momentum residual of the solid
 * cells times the cell volume (summed in cell order: the reference's bits), Mz about (ibm_cx, ibm_cy), the coefficients
 * on 1/2 rho_in u_in^2 A (A = the diameter in 2-D, pi r^2 for a sphere, diameter x Lz for a 3-D cylinder). */
int fvg_ibm_loads(fvg_run* run, double* loads);

/* The state of a moving immersed body in the layout of the reference's checkpoint key body_pose
 * (Simulation::body_checkpoint / restore_body_from_checkpoint, cpp/src/SimulationRestart.cpp:87-160): the pose the geometry
 * was built at (x, y, angle), the state of a body driven by the flow (x, y, u, v, ax, ay, dt; zeros in prescribed motion),
 * on a 3-D mesh then (z of the geometry, z, w, az), with a driven rotation (ibm_inertia > 0) then (angle, angular velocity,
 * angular acceleration) and on a 3-D mesh (omega_x, omega_y and their accelerations): 10, 13, 14 or 21 doubles.
 * fvg_get_body_state: *n = the count (0 without a moving body); with v non-NULL, *n on entry is v's capacity.
 * fvg_set_body_state: restores the body and builds its geometry at the stored pose (set the run's time first: a body in
 * prescribed motion takes its rotation at that time); a count other than the run's is FVG_ERR_ARGUMENT, a run without a
 * moving body FVG_ERR_CONFIG. */
int fvg_get_body_state(const fvg_run* run, double* v, int* n);
int fvg_set_body_state(fvg_run* run, const double* v, int n);

/* The monitor of the run's current state: out[4] = {mass, kinetic_energy, total_energy, enstrophy}. The first three are
 * the volume averages of rho, 1/2 |m|^2 / rho and rho E that the reference writes in its monitor file
 * (Simulation::volume_averages and monitor_row, cpp/src/SimulationRun.cpp:44-64, 87-90). order 0 adds the cells in the
 * reference's order (one device thread, cell by cell: its bits; about 5 ns per cell), order 1 in a fixed parallel
 * order (CTA sums in a tree, then the CTAs in order: deterministic, within rounding of the reference's). The enstrophy
 * (no counterpart in the solver; the definition of the reference's validation scripts, cases/validation/benchmarks/
 * spectra_application.py:61-67) is 1/2 the volume average of |curl u|^2, u = m / rho, with central differences over 2h,
 * wrapped across a periodic axis and one-sided at the ends of any other; w_z only on a 2-D mesh. A part of a decomposed
 * mesh is refused (its ghost planes are not the current state after a step). */
int fvg_monitor(fvg_run* run, int order, double* out);

/* Face fluxes of n face pairs (UL, UR: n x 5 doubles, axis: n ints) on the device with the run's EOS and Riemann
 * solver (RiemannSolver::face_flux, cpp/src/Schemes.cpp:202-229): F (n x 5) and the wave speeds (n). */
int fvg_face_flux_batch(fvg_run* run, const double* UL, const double* UR, const int* axis, size_t n, double* F, double* smax);

/* The residual of a state the caller keeps on the device, computed without allocating any device memory.
 *
 * No counterpart in the reference: it exists for callers that must not call cudaMalloc, such as code running inside a
 * host framework that owns every device allocation (its own caching allocator or a memory pool with a fixed budget),
 * or code that runs where the caller forbids allocation. Such a caller passes its own device buffers: U and R are nvar
 * planes of `plane` doubles each (nvar = 4 on a 2-D mesh, 5 on a 3-D mesh, the layout of fvg_device_state), R receives the
 * residual (Simulation::residual without the MUSCL-Hancock predictor, as fvg_residual with predictor_half_dt = 0) and
 * *smax (host, may be NULL) its wave speed. The work runs on cfg->device, which the call makes current on the calling
 * thread (as every entry point here does), on `stream` (NULL: the default stream); the call synchronises that stream and
 * returns when the work is done.
 *
 * The only scratch is a fixed array inside the library (about 516 KB per device, kept by every GPU that loads the library
 * until the process exits): it holds one wave-speed maximum per tile, so a mesh may have at most 65536 tiles (8x8x8 cells
 * in 3-D, 16x15 in 2-D: e.g. 320^3 or 4096 x 3840 cells). Rejected with FVG_ERR_CONFIG, besides what fvg_create rejects:
 * a mesh of more tiles, the mixed-precision form, a viscous run (its viscous residual would need a mesh-sized scratch
 * array), an immersed body, flux_quadrature = fourth, case-file source terms or time-dependent boundary values, a
 * mass-flow inlet (each needs device tables or arrays of its own). The first call on a device finds the array's device
 * address (with that device current), so make that first call before any stream capture. All calls share the array and
 * leave their results in it: calls that overlap on the GPU (other threads, other streams) race and must be serialised by
 * the caller. On failure, fvg_create_error() returns this thread's message. */
int fvg_residual_noalloc(const fvg_config* cfg, const double* U, long long plane, double* R, double* smax, void* stream);

/* ---- The learned troubled-cell sensor (no counterpart in the reference, whose WENO5-Z reconstruction, weno5z and
 * weno_line_states, cpp/src/Schemes.cpp:328-353 and 793-835, has no gate).
 *
 * A 32 -> 32 -> 32 -> 1 MLP reads a cell's 5-cell stencil along a sweep axis (25 features: rho, normal and tangential
 * velocities, p) and decides whether the cell's two reconstructions along that axis take the linear fifth-order upwind
 * values (logit below the threshold) or WENO5-Z. Weights and activations are bfloat16 on the tensor cores with float32
 * sums. The label it learns: one of the cell's two WENO5-Z face values along the axis differs from the linear
 * fifth-order upwind value there by more than tau times the quantity's physical scale at the cell (rho; the sound speed
 * for the velocities; p + p_inf). The amplitude features are taken against the same scales. Training runs on the GPU through these calls, on device buffers the caller owns:
 *   fvg_sensor_extract  features (32 floats per sample) and the departure of every (cell, axis) of a run's state
 *                       (mode 0, at index cell * dim + axis) or of the troubled ones and every keep_div-th other one
 *                       (mode 1, appended at the device counter *count up to capacity); stats (device, may be NULL):
 *                       [troubled, all] added
 *   fvg_sensor_grad     gradients (added to grad, fvg_sensor_sizes' n_params floats) and loss sum (added to *loss) of
 *                       the mean class-weighted cross-entropy (weight wpos on y = 1) over n samples
 *   fvg_sensor_adam     one Adam step of the float32 parameters (grad is cleared) and their device weights
 *   fvg_sensor_pack     device weights of float32 parameters; fvg_sensor_infer: logits of n feature rows
 * Parameter layout (floats): W1[32][32] (inputs 25..31 unused), b1[32], W2[32][32], b2[32], w3[32], b3.
 * fvg_set_sensor gates a mixed-precision WENO5-Z run with device weights (copied; NULL: plain WENO5-Z again): every
 * `every` steps (<= 0: 10) a kernel evaluates the network on every (cell, axis) of the state, the troubled set is grown by
 * `radius` cells along every axis (< 0: ceil(cfl every) + 1, the distance a wave travels until the next refresh, plus
 * one) and reduced to the stage kernels' tiles: a tile whose cells are all untroubled along an axis takes the linear
 * reconstruction for every face of that sweep. fvg_get_sensor_counts returns the (tile, axis) pairs the refreshes
 * passed to the linear reconstruction and all pairs, since the last reset.
 * Failures of the calls without a run handle: fvg_create_error(). */
int fvg_sensor_sizes(int* n_params, int* weights_bytes, int* n_inputs);
int fvg_sensor_extract(fvg_run* run, int mode, int keep_div, unsigned seed, float tau, float* X, float* departure, int* count,
                       long long capacity, unsigned long long* stats);
int fvg_sensor_grad(const void* weights, const float* X, const float* y, long long n, float wpos, float* grad, float* loss, void* stream);
int fvg_sensor_adam(float* params, float* m, float* v, float* grad, int step, float lr, float beta1, float beta2, float eps, void* weights,
                    void* stream);
int fvg_sensor_pack(const float* params, void* weights, void* stream);
int fvg_sensor_infer(const void* weights, const float* X, long long n, float* logits, void* stream);
int fvg_set_sensor(fvg_run* run, const void* weights, float threshold, int every, int radius);
int fvg_get_sensor_counts(fvg_run* run, long long* linear, long long* evaluated, int reset);
/* The gate of the last refresh, for inspection (no counterpart in the reference): cell_flags (dim x ncells bytes, axis-
 * major, cells in the reference's order; may be NULL) the network's flag of every (cell, axis), 1 = stays WENO5-Z;
 * tile_flags (dim x the tiles' count, axis-major; may be NULL) what the stage kernels read, 1 = WENO5-Z; tile (3 ints) the
 * stage tile's cells per axis and tiles (3 ints) the tiles per axis. */
int fvg_get_sensor_gate(fvg_run* run, unsigned char* cell_flags, unsigned char* tile_flags, int* tile, int* tiles);

/* ---- Batched independent problems (no counterpart in the reference, which runs one Simulation per process).
 *
 * n 2-D problems (nz = 1) of uneven sizes advance together, each with its own clock, dt and step count, as if each
 * were a run of its own: every problem's states, dt and wave speeds are the bits fvg_create + fvg_run_until give it.
 * The problems share the scheme (reconstruction, Riemann solver, time scheme Euler / SSP-RK2 / SSP-RK3, precision,
 * device) and may differ in everything else of fvg_config that a 2-D inviscid run without an immersed body uses
 * (mesh, lengths, gas, boundary conditions, limiter, cfl, dt_max). Each Runge-Kutta stage of all problems is one
 * persistent kernel launch over the tiles of the problems still running; a step's launches are captured in a CUDA graph.
 * States cross the ABI as one array: problem 0's cells, then problem 1's, ... (each in the single-run layout). */
typedef struct fvg_batch fvg_batch;
int fvg_batch_create(const fvg_config* cfgs, int n, fvg_batch** out);   /* failures: fvg_create_error() */
int fvg_batch_destroy(fvg_batch* b);
const char* fvg_batch_last_error(const fvg_batch* b);
/* the cells of all problems (the length of the state arrays below, in cells of 5 doubles) */
int fvg_batch_cells(const fvg_batch* b, long long* ncells);
int fvg_batch_upload(fvg_batch* b, const double* U, size_t ncells);
int fvg_batch_download(fvg_batch* b, double* U, size_t ncells);
/* Every problem steps from t = 0 until t >= t_end or max_steps steps (max_steps <= 0: no limit). *cell_stages (may be
 * NULL) gets the work done: the sum over problems of cells x stages per step x steps. A problem whose solution
 * diverges stops (its status 1) while the others run on; the call then returns FVG_ERR_DIVERGED. Without a schedule
 * set, the first call runs fvg_batch_autotune. */
int fvg_batch_run(fvg_batch* b, double t_end, int max_steps, long long* cell_stages);
/* problem i after a run: its time, steps taken and status (0 ok, 1 diverged) */
int fvg_batch_problem(const fvg_batch* b, int i, double* t, int* steps, int* status);
/* Autotuner: times one stage of every problem for each tile shape the library has (64x1, 128x1, 256x1, 16x15 cells)
 * and each persistent grid (1 .. the CTAs an SM holds, per SM) and keeps the fastest; returns the choice and its
 * stage time in ms. fvg_batch_set_schedule sets one by hand (ctas_per_sm 0: as many as an SM holds). */
int fvg_batch_autotune(fvg_batch* b, int* shape, int* ctas_per_sm, double* stage_ms);
int fvg_batch_set_schedule(fvg_batch* b, int shape, int ctas_per_sm);
int fvg_batch_get_schedule(const fvg_batch* b, int* shape, int* tile_x, int* tile_y, int* grid);
int fvg_batch_stream(fvg_batch* b, void** stream);
/* Kernel timing of the batched stage kernel, as fvg_set_timing / fvg_get_timing for a single run. */
int fvg_batch_set_timing(fvg_batch* b, int on);
int fvg_batch_get_timing(const fvg_batch* b, double* stage_ms, long long* stage_launches);

/* ---- The cell engine of an adaptive mesh, for meshes whose leaves are all of level 0.
 *
 * The reference's CellFluxEngine (cpp/include/fv/CellFlux.hpp:92-270: constructed from the run's EOS, RiemannSolver,
 * MusclReconstruction and BoundaryManager, then build(mesh)) and CellAdvance (cpp/include/fv/CellAdvance.hpp:27-47) on a
 * CellMesh (cpp/include/fv/CellMesh.hpp:57) given as its leaf arrays `level`, `ci`, `cj`, `ck` (CellMesh::level / ci / cj /
 * ck; ck may be NULL on a 2-D mesh). The leaves keep the caller's order: states and residuals cross the ABI as arrays of
 * nleaf leaves of 5 doubles in that order (CellMesh::U). cfg is the run's configuration (the base mesh nx x ny x nz, the
 * lengths, the scheme, the boundary conditions; the periodic axes are the periodic sides). Built: every leaf of level 0
 * (they must tile the base mesh); first order, MUSCL (every limiter), WENO3-Z, WENO5-Z; HLLC and low-Mach HLLC; the
 * boundary types but the non-reflecting outlet and the mass-flow inlet, with boundary_order 1 or 2; Euler, SSP-RK2 and
 * SSP-RK3 and MUSCL-Hancock steps; the viscous terms (2-D and 3-D) and the body force. Refused (FVG_ERR_CONFIG, message in
 * fvg_create_error()): leaves above level 0, an immersed body, sources and time-dependent boundary values,
 * positivity_fallback, the fourth-order quadrature, the mixed-precision form. */
typedef struct fvg_cells fvg_cells;
int fvg_cells_create(const fvg_config* cfg, int nleaf, const int* level, const int* ci, const int* cj, const int* ck, fvg_cells** out);
int fvg_cells_destroy(fvg_cells* e);
const char* fvg_cells_last_error(const fvg_cells* e);
/* the leaves and the faces of the mesh (CellMesh::num_leaves, CellMesh::faces.size()) */
int fvg_cells_info(const fvg_cells* e, long long* nleaf, long long* nface);
int fvg_cells_upload_state(fvg_cells* e, const double* U, size_t nleaf);
int fvg_cells_download_state(fvg_cells* e, double* U, size_t nleaf);
/* R = dU/dt of the state held (CellFluxEngine::residual, cpp/src/CellFluxResidual.cpp:1088-1105); *smax (may be NULL)
 * the largest face wave speed */
int fvg_cells_residual(fvg_cells* e, double* R, size_t nleaf, double* smax);
/* one step of length dt from time t of the state held (CellAdvance::step: with one level, the time scheme's
 * advance_fixed_dt, cpp/src/TimeScheme.cpp:100-290; MUSCL-Hancock: the leaves' limited side states predicted by dt / 2,
 * then one residual on them); *smax (may be NULL) the first stage's largest face wave speed */
int fvg_cells_step(fvg_cells* e, double dt, double t, double* smax);
/* nsteps such steps enqueued back to back (one host synchronisation at the end) */
int fvg_cells_advance(fvg_cells* e, double dt, int nsteps, double* smax);
int fvg_cells_stream(fvg_cells* e, void** stream);

#ifdef __cplusplus
}
#endif
#endif
