// Host runtime of the B200 finite-volume path and its C ABI (include/fenice_gpu.h).
//
// A run owns its device arrays (the state, a stage state, a residual / stage buffer, the viscous residual, per-CTA
// wave-speed maxima) and a control block on the device (grid.cuh: Ctl) that holds the clock, dt and the wave speeds, so
// the time loop never waits for the host: every step is a fixed sequence of kernel launches, captured once into a CUDA
// graph and replayed.
//
// Step sequences (the reference's TimeScheme::step, cpp/src/TimeScheme.cpp:110-319):
//   Euler:    [viscous] stage(U -> R) ; dt ; U = U + dt R ; end
//   SSP-RK2:  [viscous] stage(U -> R) ; dt ; Ut = U + dt R ; [viscous] stage(Ut, U0 = U -> U: 1/2 U0 + 1/2 (Ut + dt R)) ; end
//   SSP-RK3:  [viscous] stage(U -> R) ; dt ; Ut = U + dt R ; [viscous] stage(Ut, U0 = U -> R: 3/4 U0 + 1/4 (Ut + dt R)) ;
//             [viscous] stage(R, U0 = U -> U: 1/3 U0 + 2/3 (R + dt R3)) ; end
//   MUSCL-Hancock: seed (first step only: one plain residual for the wave speed) ; dt from the lagged speed ;
//             hancock(U -> Ut = U + dt R) ; end (the speed of this step is the next step's) ; the state then lives in Ut
//             (ping-pong, tracked by the host).
// "dt" reduces the CTA maxima of stage 1 into s1 and sets dt = cfl L / (s1 + 1e-10), clamped to t_end - t and dt_max;
// "end" reduces the later stages, applies check_progress, advances t and the step count and decides whether the next
// step runs (t < t_end, step limit, no error).
#include "../../include/fenice_gpu.h"
#include "expr.cuh"
#include "fourth.cuh"
#include "hancock.cuh"
#include "ibm.cuh"
#include "host_common.h"
#include "ibm_host.h"
#include "mixed_api.h"
#include "sensor.cuh"
#include "sensor_api.h"
#include "stage.cuh"
#include "tma.cuh"
#include "viscous.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

using namespace fvg;

namespace {

constexpr double kDtEps = 1e-10;   // TimeScheme.cpp:19
thread_local std::string g_create_error;

// ------------------------------------------------------------------------------------------------ control kernels
__device__ double block_reduce_max(const double* a, int n, const double* b, int nb) {
    __shared__ double red[32];
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (a[i] > v) v = a[i];
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        if (b[i] > v) v = b[i];
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w)
            if (red[w] > r) r = red[w];
    return r;
}

__device__ __forceinline__ void set_next_active(Ctl* c) {
    c->active = (c->t < c->t_end) && (c->max_steps <= 0 || c->steps < c->max_steps) && c->status == 0;
}

__global__ void k_begin(Ctl* c, double t_end, int max_steps) {
    c->t_end = t_end;
    c->max_steps = max_steps;
    c->steps = 0;
    c->status = 0;
    set_next_active(c);
}

// stage 1 of a Runge-Kutta / Euler step: its wave speed and the step dt
__global__ void k_stage1_dt(Ctl* c, const double* bm, int nb, const double* bmv, int nbv) {
    if (!c->active) return;
    const double s = block_reduce_max(bm, nb, bmv, nbv);
    if (threadIdx.x == 0) {
        c->s_stage[0] = s;
        double dt = c->cfl * c->L / (s + kDtEps);
        dt = vmin(dt, c->t_end - c->t);
        if (c->dt_max > 0.0) dt = vmin(dt, c->dt_max);
        c->dt = dt;
    }
}

__global__ void k_stage_max(Ctl* c, const int* gate, int stage, const double* bm, int nb, const double* bmv, int nbv) {
    if (!*gate) return;
    const double s = block_reduce_max(bm, nb, bmv, nbv);
    if (threadIdx.x == 0) c->s_stage[stage] = s;
}

// check_progress (cpp/src/SimulationInternal.hpp:259-267), t += dt, and whether the next step runs
__device__ void finish_step(Ctl* c, double s) {
    c->s_step = s;
    if (!(isfinite(s) && isfinite(c->dt) && c->t + c->dt > c->t)) {
        c->status = 1;
        c->active = 0;
        return;
    }
    c->t = c->t + c->dt;
    c->steps += 1;
    set_next_active(c);
}

// end of a Runge-Kutta / Euler step with `nstages` stages: S = max(s1, max(s2, s3))
__global__ void k_end_rk(Ctl* c, int nstages) {
    if (!c->active) return;
    double s = c->s_stage[0];
    if (nstages == 2) s = vmax(c->s_stage[0], c->s_stage[1]);
    if (nstages == 3) s = vmax(c->s_stage[0], vmax(c->s_stage[1], c->s_stage[2]));
    finish_step(c, s);
}

// MUSCL-Hancock (MusclHancock::step, TimeScheme.cpp:296-319)
__global__ void k_hancock_begin(Ctl* c) { c->seed = c->active && !(c->s_lag > 0.0); }
__global__ void k_hancock_seed(Ctl* c, const double* bm, int nb, const double* bmv, int nbv) {
    if (!c->seed) return;
    const double s = block_reduce_max(bm, nb, bmv, nbv);
    if (threadIdx.x == 0) c->s_lag = s;
}
__global__ void k_hancock_dt(Ctl* c) {
    if (!c->active) return;
    double dt = c->cfl * c->L / (c->s_lag + kDtEps);
    dt = vmin(dt, c->t_end - c->t);
    if (c->dt_max > 0.0) dt = vmin(dt, c->dt_max);
    c->dt = dt;
    c->half_dt = 0.5 * dt;
}
// the step's speed: the Hancock residual's, max the viscous bound (Simulation.cpp:1038-1041), lagged to the next step
__global__ void k_hancock_end(Ctl* c, const double* bm, int nb, const double* bmv, int nbv) {
    if (!c->active) return;
    const double s = block_reduce_max(bm, nb, bmv, nbv);
    if (threadIdx.x == 0) {
        c->s_lag = s;
        finish_step(c, s);
    }
}

// BoundaryManager::apply_side's mass-flow target (Boundaries.cpp:284-294), one block per side: the mean over the side's
// cells (in cell order, a sequential sum as the reference's) of cons_to_prim's density, rho_avg = max(mean, 1e-5),
// u_target = rho_in u_in / rho_avg. Other sides return at once.
template <int NV>
__global__ void __launch_bounds__(1024) k_massflow(Mesh m, Bc bc, const double* U, double rho_in, double u_in, double* u_target, const int* gate) {
    __shared__ double rho[1024];
    const int side = blockIdx.x;
    if (!*gate || bc.type[side] != kBcMassflowInlet) return;
    const int axis = side >> 1, hi = side & 1;
    const long long nx = m.nx, ny = m.ny, nz = m.nz;
    const long long count = axis == 0 ? ny * nz : (axis == 1 ? nx * nz : nx * ny);
    double sum = 0.0;
    for (long long base = 0; base < count; base += blockDim.x) {
        const long long k = base + threadIdx.x;
        if (k < count) {   // Mesh::boundary_cell (Core.hpp:136-145)
            const long long cell = axis == 0 ? k * nx + (hi ? nx - 1 : 0)
                                   : axis == 1 ? ((k / nx) * ny + (hi ? ny - 1 : 0)) * nx + k % nx
                                               : (hi ? (nz - 1) * ny * nx : 0) + k;
            rho[threadIdx.x] = vmax(read_state<NV>(bc, U, m.plane, cell)[0], Num<double>::eos_eps);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const long long lim = count - base < blockDim.x ? count - base : blockDim.x;
            for (long long q = 0; q < lim; ++q) sum = sum + rho[q];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double rin = bc.tv ? bc.tv[2] : rho_in, uin = bc.tv ? bc.tv[0] : u_in;   // at the stage time when they vary
        u_target[side] = (rin * uin) / vmax(sum / (double)count, 1e-5);
    }
}

// ---- case-file expressions (expr.h): the programs of a run on the device
struct ExprArgs {
    const expr::Op* code;
    const double* pool;
    int src[5];   // entries of source_rho, source_mx, source_my, source_E, source_mz
    int bnd[4];   // entries of u_in, v_in, rho_in, p_out as functions of t (-1: constant)
};

// TimeScheme::stage_time of the residual about to be taken (kind 0: t, 1: t + dt, 2: t + 0.5 dt, 3: `at`, 4: t +
// half_dt; TimeScheme.cpp:111-306), and Simulation::update_boundary_values at that time (Simulation.cpp:170-185): the
// time-dependent values into tv (x = y = z = 0, as compile_time_expression binds them). A value that is not finite, or
// rho_in or p_out not positive, stops the run (status 3; the reference throws).
__global__ void k_stage_values(Ctl* c, const int* gate, int kind, double at, ExprArgs x, double* tv) {
    if (!*gate) return;
    const double t = kind == 0 ? c->t : kind == 1 ? c->t + c->dt : kind == 2 ? c->t + 0.5 * c->dt : kind == 3 ? at : c->t + c->half_dt;
    c->stage_t = t;
    if (!tv) return;
    bool ok = true;
    for (int k = 0; k < 4; ++k)
        if (x.bnd[k] >= 0) {
            const double v = expr::run(x.code, x.pool, x.bnd[k], 0.0, 0.0, 0.0, t);
            tv[k] = v;
            ok = ok && isfinite(v);
        }
    if (!ok || !(tv[2] > 0.0) || !(tv[3] > 0.0)) {
        c->status = 3;
        c->active = 0;
    }
}

// evaluate_source (cpp/src/CaseFile.cpp:879-890) on the device: the five source expressions at the cell centres
// ((i + 1/2) dx, ...; z = 0 on a 2-D mesh; Mesh::xc, cpp/include/fv/Core.hpp:98-102) and the stage time, into planes
// in the state's layout. A part's own planes along the split axis and `lo` / `hi` ghost planes beyond them, at their
// places in the whole mesh of nsplit planes (wrapped across a periodic end).
template <int NV>
__global__ void k_source_field(Mesh m, ExprArgs x, const Ctl* c, const int* gate, int split, int first, int lo, int hi, int nsplit, double* S) {
    if (!*gate) return;
    const double t = c->stage_t;
    const long long nloc = split == 2 ? m.nz : m.ny;
    const long long area = split == 2 ? (long long)m.nx * m.ny : m.nx;
    const long long total = (nloc + lo + hi) * area;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long pl = e / area - lo, rem = e % area;
        long long gp = first + pl;
        if (gp < 0) gp += nsplit;
        else if (gp >= nsplit) gp -= nsplit;
        const long long i = split == 2 ? rem % m.nx : rem, j = split == 2 ? rem / m.nx : gp, k = split == 2 ? gp : 0;
        const double xc = ((double)i + 0.5) * m.dx, yc = ((double)j + 0.5) * m.dy, zc = NV == 5 ? ((double)k + 0.5) * m.dz : 0.0;
        const long long cell = pl * area + rem;
#pragma unroll 1
        for (int q = 0; q < NV; ++q) S[q * m.plane + cell] = expr::run(x.code, x.pool, x.src[q], xc, yc, zc, t);
    }
}

// ---- the monitor (fvg_monitor): volume averages of rho, the kinetic energy and rho E, and the enstrophy
// Simulation::volume_averages (cpp/src/SimulationRun.cpp:44-64) in its own order: one thread adds the cells in cell order,
// kinetic energy 0.5 (m_x^2 + m_y^2 + m_z^2) / rho (m_z = +0 on a 2-D mesh, whose terms are exact zeros), then each sum / n
__global__ void k_monitor_seq(const double* __restrict__ U, long long plane, long long n, int nvar, double* out) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (long long c = 0; c < n; ++c) {
        const double r = U[c], mx = U[plane + c], my = U[2 * plane + c], e = U[3 * plane + c];
        const double mz = nvar == 5 ? U[4 * plane + c] : 0.0;
        s0 += r;
        s1 += 0.5 * (mx * mx + my * my + mz * mz) / r;
        s2 += e;
    }
    out[0] = s0 / (double)n;
    out[1] = s1 / (double)n;
    out[2] = s2 / (double)n;
}

// the velocity component q (1, 2 or 4: u, v, w) of cell (i, j, k), and its central difference along axis d: (f(+1) - f(-1))
// / (2 h), wrapped across a periodic axis, one-sided (over h) at the two ends of any other axis
__device__ __forceinline__ double mon_vel(const double* __restrict__ U, const Mesh& m, int q, int i, int j, int k) {
    const long long c = ((long long)k * m.ny + j) * m.nx + i;
    return U[q * m.plane + c] / U[c];
}
__device__ __forceinline__ double mon_diff(const double* __restrict__ U, const Mesh& m, const int* periodic, int q, int d, int i, int j, int k) {
    const int n3[3] = {m.nx, m.ny, m.nz};
    const double h = d == 0 ? m.dx : (d == 1 ? m.dy : m.dz);
    int lo[3] = {i, j, k}, hi[3] = {i, j, k};
    lo[d] -= 1;
    hi[d] += 1;
    double span = 2.0;
    if (periodic[d]) {
        lo[d] = (lo[d] + n3[d]) % n3[d];
        hi[d] = hi[d] % n3[d];
    } else {
        if (lo[d] < 0) lo[d] = 0, span -= 1.0;
        if (hi[d] >= n3[d]) hi[d] = n3[d] - 1, span -= 1.0;
        if (span <= 0.0) return 0.0;
    }
    return (mon_vel(U, m, q, hi[0], hi[1], hi[2]) - mon_vel(U, m, q, lo[0], lo[1], lo[2])) / (span * h);
}

// per CTA: the sums of rho, the kinetic energy, rho E and 1/2 |curl u|^2 over a grid-stride share of the cells (one
// thread's cells in order, then the CTA's threads in a fixed tree: deterministic); partial[4 * blockIdx.x + q]
template <int NT>
__global__ void __launch_bounds__(NT) k_monitor_cells(Mesh m, const double* __restrict__ U, int nvar, int per0, int per1, int per2, double* partial) {
    __shared__ double red[4][NT];
    const int periodic[3] = {per0, per1, per2};
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long c = blockIdx.x * (long long)NT + threadIdx.x; c < m.ncells; c += (long long)gridDim.x * NT) {
        const int i = (int)(c % m.nx), j = (int)((c / m.nx) % m.ny), k = (int)(c / ((long long)m.nx * m.ny));
        const double r = U[c], mx = U[m.plane + c], my = U[2 * m.plane + c], e = U[3 * m.plane + c];
        const double mz = nvar == 5 ? U[4 * m.plane + c] : 0.0;
        s[0] += r;
        s[1] += 0.5 * (mx * mx + my * my + mz * mz) / r;
        s[2] += e;
        // vorticity (w_x, w_y, w_z) = (dw/dy - dv/dz, du/dz - dw/dx, dv/dx - du/dy); a 2-D mesh has w_z only
        const double wz = mon_diff(U, m, periodic, 2, 0, i, j, k) - mon_diff(U, m, periodic, 1, 1, i, j, k);
        double w2 = wz * wz;
        if (nvar == 5) {
            const double wx = mon_diff(U, m, periodic, 4, 1, i, j, k) - mon_diff(U, m, periodic, 2, 2, i, j, k);
            const double wy = mon_diff(U, m, periodic, 1, 2, i, j, k) - mon_diff(U, m, periodic, 4, 0, i, j, k);
            w2 = wx * wx + wy * wy + w2;
        }
        s[3] += 0.5 * w2;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) red[q][threadIdx.x] = s[q];
    __syncthreads();
    for (int w = NT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
#pragma unroll
            for (int q = 0; q < 4; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 4) partial[4 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}
// the CTAs' partial sums in CTA order, then / n; order 1 also takes the three volume averages from them (else k_monitor_seq
// has written them)
__global__ void k_monitor_final(const double* partial, int nblocks, long long n, int all, double* out) {
    if (threadIdx.x != 0) return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < nblocks; ++b)
        for (int q = 0; q < 4; ++q) s[q] += partial[4 * b + q];
    for (int q = all ? 0 : 3; q < 4; ++q) out[q] = s[q] / (double)n;
}

// ---- parts of a slab-decomposed mesh
// the largest of a stage's per-CTA speeds (and viscous bounds) into a slot the hosts all-reduce (0 when the gate is off)
__global__ void k_part_local(const int* gate, const double* bm, int nb, const double* bmv, int nbv, double* out) {
    if (!*gate) {
        if (threadIdx.x == 0) *out = 0.0;
        return;
    }
    const double s = block_reduce_max(bm, nb, bmv, nbv);
    if (threadIdx.x == 0) *out = s;
}
// stage 1 of a step with the all-reduced speed: dt as k_stage1_dt
__global__ void k_part_dt(Ctl* c, const double* s) {
    if (!c->active) return;
    c->s_stage[0] = s[0];
    double dt = c->cfl * c->L / (s[0] + kDtEps);
    dt = vmin(dt, c->t_end - c->t);
    if (c->dt_max > 0.0) dt = vmin(dt, c->dt_max);
    c->dt = dt;
}
__global__ void k_part_stages(Ctl* c, const double* s, int from, int n) {
    if (!c->active) return;
    for (int k = 0; k < n; ++k) c->s_stage[from + k] = s[k];
}
__global__ void k_part_seed(Ctl* c, const double* s) {
    if (c->seed) c->s_lag = s[0];
}
__global__ void k_part_hancock_end(Ctl* c, const double* s) {
    if (!c->active) return;
    c->s_lag = s[0];
    finish_step(c, s[0]);
}
// the part's `depth` first and last planes of every variable into the send buffers ([nvar][depth * area] each), or the
// receive buffers into the ghost planes before and after (an interface side only)
__global__ void k_part_pack(const double* U, long long plane, long long area, int depth, int count, int nvar, double* lo, double* hi, int do_lo,
                            int do_hi) {
    const long long n = (long long)depth * area, total = n * nvar;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
        const long long q = x / n, r = x - q * n;
        if (do_lo) lo[x] = U[q * plane + r];
        if (do_hi) hi[x] = U[q * plane + (long long)(count - depth) * area + r];
    }
}
__global__ void k_part_unpack(double* U, long long plane, long long area, int depth, int count, int nvar, const double* lo, const double* hi, int do_lo,
                              int do_hi) {
    const long long n = (long long)depth * area, total = n * nvar;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
        const long long q = x / n, r = x - q * n;
        if (do_lo) U[q * plane - n + r] = lo[x];
        if (do_hi) U[q * plane + (long long)count * area + r] = hi[x];
    }
}

// out = a + dt b over the state planes (TimeScheme.cpp:27-59: axpy)
__global__ void k_axpy(const Ctl* c, double* out, const double* a, const double* b, long long plane, long long n, int nvar) {
    if (!c->active) return;
    const double dt = c->dt;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n * nvar; e += (long long)gridDim.x * blockDim.x) {
        const long long q = e / n, i = e % n;
        const long long x = q * plane + i;
        out[x] = a[x] + dt * b[x];
    }
}

// ---- positivity_fallback (Simulation.cpp:545-584, TimeScheme.cpp:86-90)
// axpy gated by a repair flag (the control block's dt)
__global__ void k_axpy_gated(const int* gate, const Ctl* c, double* out, const double* a, const double* b, long long plane, long long n, int nvar) {
    if (!*gate) return;
    const double dt = c->dt;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n * nvar; e += (long long)gridDim.x * blockDim.x) {
        const long long q = e / n, i = e % n;
        const long long x = q * plane + i;
        out[x] = a[x] + dt * b[x];
    }
}
// the accepted candidate into the state
__global__ void k_copy_planes(const Ctl* c, double* out, const double* in, long long plane, long long n, int nvar) {
    if (!c->active) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n * nvar; e += (long long)gridDim.x * blockDim.x) {
        const long long q = e / n, i = e % n;
        out[q * plane + i] = in[q * plane + i];
    }
}
// the guard's mark: a cell of the candidate without density (rho > 0 fails, NaN included) or pressure (p + p_inf > 0
// fails, from the internal energy E - |m|^2 / (2 rho)) that is not flagged yet is flagged, and *grew set
template <int NV>
__global__ void k_fb_mark(const Ctl* c, Eos<double> e, const double* U, long long plane, long long n, unsigned char* flags, int* grew) {
    if (!c->active) return;
    const double p_inf = e.type == kIdeal ? 0.0 : e.p_inf;
    int mine = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double rho = U[i];
        bool bad = !(rho > 0.0);
        if (!bad) {
            const double m1 = U[plane + i], m2 = U[2 * plane + i], m3 = NV == 5 ? U[4 * plane + i] : 0.0;
            const double ke = 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / rho;
            bad = !(pressure(e, U[3 * plane + i] - ke) + p_inf > 0.0);
        }
        if (bad && !flags[i]) {
            flags[i] = 1;
            mine = 1;
        }
    }
    if (__syncthreads_or(mine) && threadIdx.x == 0) atomicExch(grew, 1);
}

// reference layout (cells of 5 doubles) <-> state planes; a 2-D mesh carries no rho w (it must be zero)
__global__ void k_aos_to_planes(const double* aos, double* U, long long plane, long long n, int nvar, int* bad) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        for (int q = 0; q < nvar; ++q) U[q * plane + c] = aos[5 * c + q];
        if (nvar == 4 && aos[5 * c + 4] != 0.0) atomicOr(bad, 1);
    }
}
__global__ void k_planes_to_aos(const double* U, double* aos, long long plane, long long n, int nvar) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        for (int q = 0; q < 5; ++q) aos[5 * c + q] = q < nvar ? U[q * plane + c] : 0.0;
    }
}

template <int RIEMANN, int NV>
__global__ void k_face_flux(Eos<double> e, double shock_blend, const double* UL, const double* UR, const int* axis, long long n, double* F, double* sm) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        St<double, NV> ul, ur, f;
        for (int q = 0; q < NV; ++q) {
            ul[q] = UL[5 * k + q];
            ur[q] = UR[5 * k + q];
        }
        sm[k] = face_flux<RIEMANN>(e, shock_blend, ul, ur, axis[k], f);
        for (int q = 0; q < NV; ++q) F[5 * k + q] = f[q];
    }
}

// Simulation::ibm_loads (cpp/src/SimulationRun.cpp:134-155): {Fx, Fy, Mz} = the momentum residual of the solid cells times
// the cell volume, summed in cell order (one thread: the reference's order, so the bits), Mz about (cx, cy).
__global__ void k_ibm_loads(const double* R, const double* U, long long plane, const int* cells, int n, double vol, int nx, int ny, double dx,
                            double dy, double cx, double cy, double gx, double gy, int grav, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double fx = 0.0, fy = 0.0, mz = 0.0;
    for (int k = 0; k < n; ++k) {
        const int c = cells[k];
        double rx = R[plane + c], ry = R[2 * plane + c];
        if (grav) {   // the weight is not a load
            rx -= U[c] * gx;
            ry -= U[c] * gy;
        }
        const double ex = rx * vol, ey = ry * vol;
        fx += ex;
        fy += ey;
        const double xc = ((c % nx) + 0.5) * dx + 0.0, yc = (((c / nx) % ny) + 0.5) * dy + 0.0;
        mz += (xc - cx) * ey - (yc - cy) * ex;
    }
    out[0] = fx;
    out[1] = fy;
    out[2] = mz;
}

// ------------------------------------------------------------------------------------------------ kernel dispatch
// Simulation::ibm_load_terms + sum_load_terms (cpp/src/SimulationRun.cpp:312-350) of the first stage's residual R: per
// solid cell (in cell order, one thread: the reference's sums) the momentum residual times the cell volume, its moment
// about the pivot, and in 3-D the z component and the moments about x and y; out = {fx, fy, mz, fz, mx, my}.
__global__ void k_body_loads(const int* gate, const double* R, const double* U, long long plane, const int* cells, int n, double vol, int nx, int ny,
                             double dx, double dy, double dz, int three_d, double px, double py, double pz, int grav, double gx, double gy, double gz,
                             double* out) {
    if (!*gate || threadIdx.x != 0) return;
    double fx = 0.0, fy = 0.0, mz = 0.0, fz = 0.0, mx = 0.0, my = 0.0;
    for (int q = 0; q < n; ++q) {
        const long long c = cells[q];
        double rx = R[plane + c], ry = R[2 * plane + c];
        if (grav) {   // the weight is not a load
            rx -= U[c] * gx;
            ry -= U[c] * gy;
        }
        const double ex = rx * vol, ey = ry * vol;
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
        const double xc = (i + 0.5) * dx + 0.0, yc = (j + 0.5) * dy + 0.0;
        double ez = 0.0, tx = 0.0, ty = 0.0;
        if (three_d) {
            double rz = R[4 * plane + c];
            if (grav) rz -= U[c] * gz;
            ez = rz * vol;
            const double x = xc - px, y = yc - py, z = (k + 0.5) * dz + 0.0 - pz;
            tx = y * ez - z * ey;
            ty = z * ex - x * ez;
        }
        fx += ex;
        fy += ey;
        mz += (xc - px) * ey - (yc - py) * ex;
        fz += ez;
        mx += tx;
        my += ty;
    }
    out[0] = fx;
    out[1] = fy;
    out[2] = mz;
    out[3] = fz;
    out[4] = mx;
    out[5] = my;
}

template <int DIM> struct Tile;
// 3-D: 256 threads per 8x8x8 tile, two CTAs per SM (at most 120 registers, 101 KB of shared memory): 16 warps per SM;
// measured at 256^3 (WENO5-Z, low-Mach HLLC): 11.07 ms per launch against 12.60 with 192 threads, the same bits
template <> struct Tile<3> { static constexpr int X = 8, Y = 8, Z = 8, NT = 256; };
template <> struct Tile<2> { static constexpr int X = 16, Y = 15, Z = 1, NT = 256; };

// Each kernel gets its shared-memory limit raised once, when a run is created (never during a graph capture).
template <int DIM, int RECON, int RIEMANN, bool FULL> struct StageK {
    using Tl = Tile<DIM>;
    using S = StageShape<DIM, RECON, Tl::X, Tl::Y, Tl::Z>;
    static cudaError_t prepare() {
        return cudaFuncSetAttribute(stage_kernel<DIM, RECON, RIEMANN, Tl::X, Tl::Y, Tl::Z, Tl::NT, FULL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)S::SMEM_BYTES);
    }
    static cudaError_t launch(const StageArgs& a, int nblocks, cudaStream_t s) {
        stage_kernel<DIM, RECON, RIEMANN, Tl::X, Tl::Y, Tl::Z, Tl::NT, FULL><<<nblocks, Tl::NT, S::SMEM_BYTES, s>>>(a);
        return cudaGetLastError();
    }
};

struct StageLauncher {
    cudaError_t (*prepare)() = nullptr;
    cudaError_t (*launch)(const StageArgs&, int, cudaStream_t) = nullptr;
};

template <int DIM, int RECON, bool FULL> StageLauncher stage_launcher_r(int riemann) {
    if (riemann == kLowMach) return {StageK<DIM, RECON, kLowMach, FULL>::prepare, StageK<DIM, RECON, kLowMach, FULL>::launch};
    return {StageK<DIM, RECON, kHLLC, FULL>::prepare, StageK<DIM, RECON, kHLLC, FULL>::launch};
}

template <int DIM, bool FULL> StageLauncher stage_launcher_f(int recon, int riemann) {
    switch (recon) {
    case kFirstOrder: return stage_launcher_r<DIM, kFirstOrder, FULL>(riemann);
    case kMuscl: return stage_launcher_r<DIM, kMuscl, FULL>(riemann);
    case kWeno3: return stage_launcher_r<DIM, kWeno3, FULL>(riemann);
    default: return stage_launcher_r<DIM, kWeno5, FULL>(riemann);
    }
}

// full: the run has a part interface, a non-reflecting side, the positivity fallback or the body force (the stage
// kernels with their code); else the lean instantiation
template <int DIM> StageLauncher stage_launcher(int recon, int riemann, bool full) {
    return full ? stage_launcher_f<DIM, true>(recon, riemann) : stage_launcher_f<DIM, false>(recon, riemann);
}

// the 3-D viscous sweep: 8x8x8 tiles, 384 threads (two CTAs per SM by shared memory, 24 warps; 3.13 ms per launch at
// 256^3 against 4.76 with 192 threads, the same bits)
constexpr int kViscNT = 384;
cudaError_t prepare_viscous() {
    return cudaFuncSetAttribute(viscous_kernel<8, 8, 8, kViscNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ViscShape<8, 8, 8>::SMEM_BYTES);
}
cudaError_t launch_viscous(const ViscArgs& a, int nblocks, cudaStream_t s) {
    viscous_kernel<8, 8, 8, kViscNT><<<nblocks, kViscNT, ViscShape<8, 8, 8>::SMEM_BYTES, s>>>(a);
    return cudaGetLastError();
}
// the 2-D sweep: 16 x 16 tiles, 256 threads (the mixed form uses it too: the FP32 viscous kernel is 3-D only)
constexpr int kVisc2T = 16;
cudaError_t prepare_viscous2d() {
    return cudaFuncSetAttribute(viscous2d_kernel<kVisc2T, kVisc2T, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)Visc2Shape<kVisc2T, kVisc2T>::SMEM_BYTES);
}
cudaError_t launch_viscous2d(const ViscArgs& a, int nblocks, cudaStream_t s) {
    viscous2d_kernel<kVisc2T, kVisc2T, 256><<<nblocks, 256, Visc2Shape<kVisc2T, kVisc2T>::SMEM_BYTES, s>>>(a);
    return cudaGetLastError();
}

// MUSCL-Hancock tiles: 16 x 16 in 2-D, 8 x 8 x 4 in 3-D (93 KB of shared memory: two CTAs per SM); FULL as the stage kernels
template <int RIEMANN, bool FULL> cudaError_t prepare_hancock_t(int dim) {
    if (dim == 3)
        return cudaFuncSetAttribute(hancock3d_kernel<RIEMANN, 8, 8, 4, 256, FULL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Hancock3Shape<8, 8, 4>::SMEM_BYTES);
    return cudaFuncSetAttribute(hancock_kernel<RIEMANN, 16, 16, 256, FULL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)HancockShape<16, 16>::SMEM_BYTES);
}
template <int RIEMANN, bool FULL> cudaError_t launch_hancock_t(int dim, const HancockArgs& a, int nblocks, cudaStream_t s) {
    if (dim == 3)
        hancock3d_kernel<RIEMANN, 8, 8, 4, 256, FULL><<<nblocks, 256, Hancock3Shape<8, 8, 4>::SMEM_BYTES, s>>>(a);
    else
        hancock_kernel<RIEMANN, 16, 16, 256, FULL><<<nblocks, 256, HancockShape<16, 16>::SMEM_BYTES, s>>>(a);
    return cudaGetLastError();
}
cudaError_t prepare_hancock(int riemann, bool full, int dim) {
    if (riemann == kLowMach) return full ? prepare_hancock_t<kLowMach, true>(dim) : prepare_hancock_t<kLowMach, false>(dim);
    return full ? prepare_hancock_t<kHLLC, true>(dim) : prepare_hancock_t<kHLLC, false>(dim);
}

}   // namespace

// ------------------------------------------------------------------------------------------------ the run
struct fvg_run {
    fvg_config cfg{};
    std::string err;
    int dim = 2, nvar = 4;
    Mesh m{};
    Bc bc{};
    Eos<double> eos{};
    double L = 0.0;
    cudaStream_t stream = nullptr;
    double *U = nullptr, *Ut = nullptr, *R = nullptr, *Rv = nullptr, *staging = nullptr;
    double* bm[3] = {nullptr, nullptr, nullptr};
    double* bmv[3] = {nullptr, nullptr, nullptr};
    double* bm_seed = nullptr;
    Ctl* ctl = nullptr;
    int tiles[3] = {1, 1, 1}, nb = 0, ntiles_v[3] = {1, 1, 1}, nbv = 0, ntiles_h[3] = {1, 1, 1}, nbh = 0;
    StageLauncher stage;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};   // two steps, by the buffer the state starts in (MUSCL-Hancock ping-pong)
    int cur = 0;   // MUSCL-Hancock ping-pong: 0 the state is in U, 1 in Ut
    // kernel timing (fvg_set_timing): CUDA events around each launch of the stage (or predictor) kernel and of the
    // viscous kernel, on the run's stream; the steps are then launched one by one instead of as graphs
    struct EvTimer {
        std::vector<cudaEvent_t> ev;
        size_t used = 0;
        std::vector<size_t> step_start;   // ev index at the start of each step enqueued since the last flush
        double ms = 0.0;
        long long n = 0;
    };
    bool timing = false;
    EvTimer t_stage, t_visc;
    // immersed body (use_ibm): the mask, the forced-state slots and buffer, the ghost table, the deep solid cells
    bool ibm = false;
    int ng = 0, nd = 0;
    unsigned char* d_mask = nullptr;
    int *d_slot = nullptr, *d_ghost = nullptr, *d_img_cell = nullptr, *d_deep = nullptr;
    int* d_solid = nullptr;   // the solid cells in cell order (the loads' sum)
    int nsolid = 0;
    double* d_loads = nullptr;
    double *d_forced = nullptr, *d_img_w = nullptr, *d_ratio = nullptr, *d_gn = nullptr, *d_span = nullptr;
    // the learned sensor (fvg_set_sensor): its weights (a copy), the logit threshold, the refresh period and dilation,
    // the network's flags of every (cell, axis), the tile flags the stage kernels read, the counters
    void* sens = nullptr;
    float sens_theta = 0.0f;
    int sens_every = 5, sens_radius = 4;
    unsigned char* sens_flags = nullptr;
    unsigned char* sens_tiles = nullptr;   // per axis and stage tile
    unsigned long long* sens_count = nullptr;
    // one part of a slab-decomposed mesh (fvg_create_part): the split axis (z in 3-D, y in 2-D), the part's first plane
    // and plane count, the ghost depth, which sides are interfaces with a neighbouring part, the offset of the first
    // interior plane in the state arrays (U, Ut, R, Rv point there), the exchange buffers (send lo / hi, recv lo / hi:
    // depth x plane cells x nvar each) and the all-reduce slots
    double* d_utarget = nullptr;   // mass-flow inlets: the target velocity per side (Bc::u_target)
    unsigned char* fb_flags = nullptr;   // positivity_fallback: the cells flagged in the current stage
    int* fb_grew = nullptr;              // and whether the last mark flagged a new one (the repeat's gate)
    bool full = false;   // the kernels with the code of part interfaces, NRBC, the fallback, the body force
    bool is_part = false;
    int nparts = 1, part = 0, split = 2, first = 0, count = 0, depth = 0, peer[2] = {0, 0};
    long long goff = 0, area = 0, xcount = 0;
    double* xbuf = nullptr;
    double* xred = nullptr;
    int nsplit = 1;   // planes of the whole mesh along the split axis
    // case-file expressions (fvg_config source / boundary_*): the programs on the device, the source field (planes in the
    // state's layout with its ghost planes; d_src is the allocation) and the time-dependent boundary values (d_tv: 4)
    ExprArgs xa{};
    expr::Op* d_code = nullptr;
    double* d_pool = nullptr;
    bool src_on = false, src_unsteady = false, tv_on = false;
    double* d_src = nullptr;
    double* d_tv = nullptr;
    // a moving immersed body (prescribed motion): the pose (displacement and velocities), the pose the geometry was built
    // at, the host tables of that geometry, the wall velocities on the device (per ghost / deep cell)
    struct Pose {
        double x = 0.0, y = 0.0, z = 0.0, w = 0.0, angle = 0.0, u = 0.0, v = 0.0, omega = 0.0, omega_x = 0.0, omega_y = 0.0;
    };
    bool moving = false, dynamic = false;
    Pose pose, built;
    // a body driven by the flow (Simulation::BodyDynamics): its state, the centre of mass from the pivot, the loads of the
    // first stage of the step on the device (6: fx, fy, mz, fz, mx, my)
    struct Body {
        double x = 0, y = 0, u = 0, v = 0, z = 0, w = 0, az = 0, ax = 0, ay = 0, dt = 0, fx = 0, fy = 0, fz = 0;
        double th = 0, om = 0, aom = 0, mx = 0, my = 0, mz = 0, omx = 0, omy = 0, aomx = 0, aomy = 0;
    } body;
    double cm0[2] = {0.0, 0.0};
    double* d_bload = nullptr;
    // fvg_monitor: per-CTA partial sums (4 per CTA) and the four results (allocated at the first call)
    double* d_mon = nullptr;
    // TMA tensor maps of U, Ut and R for the stage kernels that stage their interior tiles by TMA (tma_on: built)
    TmaMaps tma[3];
    bool tma_on = false;
    // a section body: its vertices where it was placed at t = 0 (the reference the poses turn about the pivot), and how far
    // a vertex lies from the pivot (ImmersedBoundary::enable_motion's reach)
    std::vector<double> ref_poly;
    double reach = 0.0;
    IbmTable tab;
    double *d_gvel = nullptr, *d_dvel = nullptr;
    // flux_quadrature = fourth: the face arrays of the face passes (fourth.cuh; one allocation, d_fourth)
    bool fourth = false;
    FourthArgs fa{};
    void* d_fourth = nullptr;
    // fvg_step_host: the copy stream, the events of the slabs' uploads and downloads, and the steps it took with the
    // sensor on (the sensor's refresh cadence across calls)
    cudaStream_t xfer = nullptr;
    std::vector<cudaEvent_t> ev_host;
    long long host_steps = 0;
    double res_time = NAN;   // fvg_set_stage_time (NaN: the run's time)
    int res_kind = -1;       // the stage-time kind residual_stage takes (-1: its stage index)
    double* Ucur() { return cur ? Ut : U; }
};

namespace {

int fail(fvg_run* r, int code, const std::string& msg) {
    r->err = msg;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(run, FVG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Whether a configuration has case-file source terms (a value that is not a whole number equal to 0: Params.cpp:280-286)
// or time-dependent boundary values (an expression that is not a whole number, or a time table).
bool has_expressions(const fvg_config& c) {
    for (int q = 0; q < 5; ++q)
        if (c.source[q]) {
            char* end = nullptr;
            const double d = std::strtod(c.source[q], &end);
            if (!(end && *end == '\0' && d == 0.0)) return true;
        }
    for (int k = 0; k < 4; ++k) {
        if (c.boundary_table[k] && c.boundary_table_rows[k] > 0) return true;
        if (c.boundary_expr[k] && *c.boundary_expr[k]) {
            char* end = nullptr;
            std::strtod(c.boundary_expr[k], &end);
            if (!(end && end != c.boundary_expr[k] && *end == '\0')) return true;
        }
    }
    return false;
}

std::string validate(const fvg_config& c) {
    if (c.nx < 1 || c.ny < 1 || c.nz < 1) return "nx, ny, nz must be >= 1";
    if (!(c.Lx > 0 && c.Ly > 0 && c.Lz > 0)) return "Lx, Ly, Lz must be > 0";
    if ((long long)c.nx * c.ny * c.nz > (1LL << 31) - 1) return "more than 2^31 - 1 cells";
    if (c.eos_type != FVG_EOS_IDEAL && c.eos_type != FVG_EOS_STIFFENED) return "unknown eos_type";
    if (!(c.gamma > 1.0)) return "gamma must be > 1";
    if (c.riemann != FVG_RIEMANN_HLLC && c.riemann != FVG_RIEMANN_LOWMACH) return "unknown riemann_solver";
    if (c.reconstruction < FVG_RECON_NONE || c.reconstruction > FVG_RECON_WENO5) return "unknown reconstruction";
    if (c.limiter < 0 || c.limiter > 3) return "unknown muscl_limiter";
    if (c.time_scheme < 0 || c.time_scheme > 3) return "unknown time_scheme";
    if (c.boundary_order != 1 && c.boundary_order != 2) return "boundary_order must be 1 or 2";
    if (c.precision != FVG_PREC_FP64 && c.precision != FVG_PREC_MIXED) return "unknown precision";
    if (c.precision == FVG_PREC_MIXED && c.reconstruction == FVG_RECON_NONE) return "the mixed-precision form needs a reconstruction (muscl, weno3, weno5)";
    if (c.precision == FVG_PREC_MIXED && c.time_scheme == FVG_TS_HANCOCK) return "the mixed-precision form runs the Runge-Kutta schemes (MUSCL-Hancock is FP64 only)";
    const int naxes = c.nz > 1 ? 3 : 2;
    for (int s = 0; s < 2 * naxes; ++s) {
        if (c.bc[s] < 0 || c.bc[s] > FVG_BC_NONREFLECTING) return "unknown boundary type";
    }
    for (int a = 0; a < naxes; ++a)
        if ((c.bc[2 * a] == FVG_BC_PERIODIC) != (c.bc[2 * a + 1] == FVG_BC_PERIODIC))
            return "a periodic axis needs both of its sides periodic";
    if (c.time_scheme == FVG_TS_HANCOCK && c.reconstruction != FVG_RECON_MUSCL) return "time_scheme = MUSCL-Hancock needs reconstruction = muscl";
    if ((c.reconstruction == FVG_RECON_WENO3 || c.reconstruction == FVG_RECON_WENO5) && c.time_scheme == FVG_TS_SSPRK2)   // Params.cpp:444-446
        return std::string("reconstruction = ") + (c.reconstruction == FVG_RECON_WENO3 ? "weno3" : "weno5") +
               " is not used with SSP Runge-Kutta 2 (use SSP Runge-Kutta 3)";
    if (!(c.weno_epsilon >= 0.0)) return "weno_epsilon must be >= 0";
    if (!(c.dt_max >= 0.0) || !std::isfinite(c.dt_max)) return "dt_max must be finite and >= 0 (0: off)";
    if (c.use_viscous && (!(c.mu >= 0.0) || !(c.pr > 0.0))) return "mu must be >= 0 and pr > 0 with use_viscous";
    if (c.use_bodyforce && c.precision == FVG_PREC_MIXED) return "the body force runs in the FP64 form only";
    if (has_expressions(c) && c.precision == FVG_PREC_MIXED)
        return "case-file source terms and time-dependent boundary values run in the FP64 form only";
    if (c.nparams < 0 || (c.nparams > 0 && (!c.param_names || !c.param_values))) return "param_names / param_values missing";
    if (c.flux_quadrature != 0 && c.flux_quadrature != 1) return "flux_quadrature must be midpoint (0) or fourth (1)";
    if (c.flux_quadrature == 1) {   // Params.cpp:450-456
        if (c.reconstruction != FVG_RECON_WENO3 && c.reconstruction != FVG_RECON_WENO5) return "flux_quadrature = fourth needs reconstruction = weno3 or weno5";
        if (c.use_ibm) return "flux_quadrature = fourth is not available with an immersed body yet";
        if (c.positivity_fallback) return "positivity_fallback needs flux_quadrature = midpoint";
        if (c.precision != FVG_PREC_FP64) return "flux_quadrature = fourth runs in the FP64 form only";
    }
    if (c.positivity_fallback) {   // Params.cpp:464-467
        if (c.reconstruction != FVG_RECON_WENO3 && c.reconstruction != FVG_RECON_WENO5)
            return "positivity_fallback needs reconstruction = weno3 or weno5 (the other schemes keep their reconstructed states between the cells)";
        if (c.precision != FVG_PREC_FP64) return "positivity_fallback runs in the FP64 form only";
    }
    if (!(c.cfl > 0)) return "cfl must be > 0";
    if (c.use_ibm) {   // a prescribed motion (Params.cpp:505-516)
        const bool moving = c.ibm_vx != 0.0 || c.ibm_vy != 0.0 || c.ibm_vz != 0.0 || c.ibm_omega != 0.0 || c.ibm_omega_x != 0.0 || c.ibm_omega_y != 0.0;
        if ((c.ibm_omega_from > 0.0 || c.ibm_omega_until > 0.0) && c.ibm_omega == 0.0 && c.ibm_omega_x == 0.0 && c.ibm_omega_y == 0.0)
            return "ibm_omega_from / ibm_omega_until need a rotation (ibm_omega)";
        if (c.ibm_omega_until > 0.0 && c.ibm_omega_until <= c.ibm_omega_from) return "ibm_omega_until must be later than ibm_omega_from";
        if (moving && c.ibm_curvature) return "ibm_curvature is not available for a moving body";
        if (moving && c.nz > 1 && c.ibm_shape != 1) return "a moving body in 3-D is a sphere (for now)";
        if (c.ibm_shape == 2 && c.ibm_mass > 0.0 && c.ibm_inertia > 0.0 && !c.ibm_cm_given)
            return "a body that translates and turns about its pivot needs the centre of mass: set ibm_cm_x and ibm_cm_y, its offset from the pivot (0 0: at the pivot)";
        if (c.nz == 1 && (c.ibm_omega_x != 0.0 || c.ibm_omega_y != 0.0)) return "ibm_omega_x and ibm_omega_y need a 3-D mesh (nz > 1)";
        if (moving && c.nz == 1 && c.ibm_vz != 0.0) return "ibm_vz needs a 3-D mesh (nz > 1)";
        // a body driven by the flow (Params.cpp:517-546)
        const bool trans = c.ibm_mass > 0.0, rot = c.ibm_inertia > 0.0;
        if (!(c.ibm_mass >= 0.0) || !(c.ibm_stiff_x >= 0.0) || !(c.ibm_stiff_y >= 0.0) || !(c.ibm_stiff_z >= 0.0) || !(c.ibm_damp_x >= 0.0) ||
            !(c.ibm_damp_y >= 0.0) || !(c.ibm_damp_z >= 0.0))
            return "ibm_mass, ibm_stiff_x/y/z and ibm_damp_x/y/z must be >= 0";
        if (!(c.ibm_inertia >= 0.0) || !(c.ibm_stiff_theta >= 0.0) || !(c.ibm_damp_theta >= 0.0))
            return "ibm_inertia, ibm_stiff_theta and ibm_damp_theta must be >= 0";
        if (!trans && (c.ibm_stiff_x != 0.0 || c.ibm_stiff_y != 0.0 || c.ibm_stiff_z != 0.0 || c.ibm_damp_x != 0.0 || c.ibm_damp_y != 0.0 || c.ibm_damp_z != 0.0))
            return "ibm_stiff_* and ibm_damp_* act on a body driven by the flow: set ibm_mass > 0";
        if (!rot && (c.ibm_stiff_theta != 0.0 || c.ibm_damp_theta != 0.0))
            return "ibm_stiff_theta and ibm_damp_theta act on a body whose rotation is driven by the flow: set ibm_inertia > 0";
        if (c.ibm_cm_given) {
            if (c.nz > 1) return "ibm_cm_x / ibm_cm_y are 2-D (a sphere turns about its centre)";
            if (!trans || !rot) return "ibm_cm_x / ibm_cm_y act on a body whose translation and rotation are both driven: set ibm_mass > 0 and ibm_inertia > 0";
            if (!(c.ibm_inertia > c.ibm_mass * (c.ibm_cm_x * c.ibm_cm_x + c.ibm_cm_y * c.ibm_cm_y)))
                return "ibm_inertia is the moment of inertia about the pivot: it must exceed ibm_mass times the squared distance of the centre of mass from it";
        }
        if (trans || rot) {
            if (!rot && (c.ibm_omega != 0.0 || c.ibm_omega_x != 0.0 || c.ibm_omega_y != 0.0))
                return "a body driven by the flow translates only unless its rotation is driven too (ibm_omega must be 0, or set ibm_inertia > 0)";
            if (rot) {
                if (c.nz > 1 && c.ibm_stiff_theta != 0.0) return "ibm_stiff_theta: a sphere has no angle to pull back (use ibm_damp_theta)";
                if (c.ibm_omega_from > 0.0 || c.ibm_omega_until > 0.0) return "ibm_omega_from / ibm_omega_until act on a prescribed rotation, not on a driven one";
                if (!trans && (c.ibm_vx != 0.0 || c.ibm_vy != 0.0 || c.ibm_vz != 0.0))
                    return "a driven rotation with a prescribed translation is not available: the body is pinned at its placement";
            }
            if (c.time_scheme == FVG_TS_HANCOCK) return "a body driven by the flow needs a Runge-Kutta or Euler time scheme (its loads come from the first stage)";
            if (c.positivity_fallback) return "a body driven by the flow with positivity_fallback is not supported on the device";
        }
    }
    // load_boundary_functions (Simulation.cpp:152-153); time-dependent ones are checked at t = 0 when compiled
    const bool rho_fn = (c.boundary_expr[2] && *c.boundary_expr[2]) || (c.boundary_table[2] && c.boundary_table_rows[2] > 0);
    const bool p_fn = (c.boundary_expr[3] && *c.boundary_expr[3]) || (c.boundary_table[3] && c.boundary_table_rows[3] > 0);
    if ((!rho_fn && !(c.rho_in > 0.0)) || (!p_fn && !(c.p_out > 0.0))) return "rho_in and p_out must be positive";
    if (!(c.nrbc_sigma >= 0.0)) return "nrbc_sigma must be >= 0";   // Params.cpp:489-490
    if (!(c.nrbc_beta <= 1.0)) return "nrbc_beta must be <= 1 (< 0: local Mach number)";
    return "";
}

// the non-reflecting outlet's parameters (BCParams, cpp/include/fv/Boundaries.hpp:23-29; length: the domain, h: the cells)
void set_nrbc(const fvg_config& c, Bc& bc) {
    bc.nrbc_sigma = c.nrbc_sigma;
    bc.nrbc_beta = c.nrbc_beta;
    bc.length[0] = c.Lx;
    bc.length[1] = c.Ly;
    bc.length[2] = c.Lz;
    bc.h[0] = c.Lx / c.nx;
    bc.h[1] = c.Ly / c.ny;
    bc.h[2] = c.Lz / c.nz;
}

// the constant body force of a configuration (Simulation::setup, cpp/src/Simulation.cpp:362-363: gz only on a 3-D mesh)
void set_body_force(const fvg_config& c, Bc& bc) {
    bc.grav_on = c.use_bodyforce ? 1 : 0;
    bc.grav[0] = c.use_bodyforce ? c.gx : 0.0;
    bc.grav[1] = c.use_bodyforce ? c.gy : 0.0;
    bc.grav[2] = c.use_bodyforce && c.nz > 1 ? c.gz : 0.0;
}

// halo kinds of the sides for a reconstruction `depth` cells deep (Simulation.cpp:868-905, 1107-1176)
void halo_kinds(const fvg_config& c, int depth, int kinds[6]) {
    const int n3[3] = {c.nx, c.ny, c.nz};
    for (int s = 0; s < 6; ++s) kinds[s] = kHaloNone;
    if (c.reconstruction == FVG_RECON_NONE) return;
    const int naxes = c.nz > 1 ? 3 : 2;
    for (int a = 0; a < naxes; ++a) {
        const bool per = c.bc[2 * a] == FVG_BC_PERIODIC && c.bc[2 * a + 1] == FVG_BC_PERIODIC;
        for (int h = 0; h < 2; ++h) {
            const int s = 2 * a + h, bt = c.bc[s];
            if (per && n3[a] >= depth)
                kinds[s] = kHaloWrap;
            else if (c.boundary_order == 2 && bt != FVG_BC_PERIODIC && bt != FVG_BC_NONREFLECTING && n3[a] >= depth)
                kinds[s] = kHaloSlab;
        }
    }
}

StageArgs stage_args(fvg_run* r, const double* Uin, const double* U0, double* out, int mode, double ca, double cb, const double* Rv, double* bm,
                     const int* gate) {
    StageArgs a{};
    a.m = r->m;
    a.bc = r->bc;
    a.eos = r->eos;
    a.shock_blend = r->cfg.shock_blend;
    a.weno_eps = r->cfg.weno_epsilon;
    a.limiter = r->cfg.limiter;
    a.mode = mode;
    a.ca = ca;
    a.cb = cb;
    a.U = Uin;
    a.U0 = U0;
    a.out = out;
    // the 3-D mixed viscous kernel keeps its FP32 balance sums in the Rv array (4 float planes in the room of 5 doubles)
    const bool f32v = Rv && r->cfg.precision == FVG_PREC_MIXED && r->dim == 3;
    a.Rv = f32v ? nullptr : Rv;
    a.Rvf = f32v ? reinterpret_cast<const float*>(Rv) : nullptr;
    a.blockmax = bm;
    a.ctl = r->ctl;
    a.gate = gate;
    for (int d = 0; d < 3; ++d) a.tiles[d] = r->tiles[d];
    a.sens_flags = r->sens ? r->sens_tiles : nullptr;
    a.tma = !r->tma_on ? nullptr : Uin == r->U ? &r->tma[0] : Uin == r->Ut ? &r->tma[1] : Uin == r->R ? &r->tma[2] : nullptr;
    return a;
}

// The TMA tensor maps of the run's state buffers U, Ut and R (tma.cuh) for the 3-D mixed WENO5-Z kernels of a whole mesh
// without an immersed body (lean kernels); cuTensorMapEncodeTiled through the runtime's driver entry point. A mesh
// whose row is not a multiple of 16 bytes (nx odd) keeps the index-mapping loader.
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
void build_tma_maps(fvg_run* r) {
    r->tma_on = false;
    const fvg_config& c = r->cfg;
    if (r->dim != 3 || c.precision != FVG_PREC_MIXED || c.reconstruction != FVG_RECON_WENO5 || r->full || r->ibm || c.use_ibm || c.nx % 2 != 0)
        return;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
        return;
    const EncodeTiled encode = reinterpret_cast<EncodeTiled>(fn);
    const cuuint64_t dims[4] = {(cuuint64_t)r->m.nx, (cuuint64_t)r->m.ny, (cuuint64_t)r->m.nz, 5};
    const cuuint64_t strides[3] = {(cuuint64_t)r->m.nx * 8, (cuuint64_t)r->m.nx * r->m.ny * 8, (cuuint64_t)r->m.plane * 8};
    const cuuint32_t boxes[5][4] = {{16, 8, 8, 5}, {8, 14, 8, 5}, {8, 8, 14, 5}, {8, 3, 8, 5}, {8, 8, 3, 5}};   // (TmaMaps)
    const cuuint32_t es[4] = {1, 1, 1, 1};
    double* bufs[3] = {r->U, r->Ut, r->R};
    for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 5; ++a)
            if (encode(&r->tma[b].m[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, bufs[b], dims, strides, boxes[a], es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                       CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return;
    r->tma_on = true;
}

ViscArgs visc_args(fvg_run* r, const double* Uin, double* bmv, const int* gate) {
    ViscArgs a{};
    a.m = r->m;
    a.bc = r->bc;
    a.eos = r->eos;
    const double g = r->cfg.gamma;
    a.mu = r->cfg.mu;
    a.k_cond = r->cfg.mu * g / (r->cfg.pr * (g - 1.0));   // TransportLaw (Core.hpp:194-197)
    a.L = r->L;
    a.inv_h2 = r->dim == 3 ? 1.0 / (r->m.dx * r->m.dx) + 1.0 / (r->m.dy * r->m.dy) + 1.0 / (r->m.dz * r->m.dz)   // inv_h2_3d
                           : 1.0 / (r->m.dx * r->m.dx) + 1.0 / (r->m.dy * r->m.dy);                               // inv_h2_2d
    a.nvar = r->nvar;
    a.u_in = r->cfg.u_in;
    a.v_in = r->cfg.v_in;
    a.bface2 = r->cfg.boundary_order == 2 && r->cfg.reconstruction != FVG_RECON_NONE;   // Params.cpp:470: first order keeps order 1
    for (int d = 0; d < 3; ++d) {   // (a split periodic axis is not wrapped in a part: its ends are interfaces)
        const bool split = r->is_part && d == r->split;
        a.periodic[d] = r->cfg.bc[2 * d] == FVG_BC_PERIODIC && r->cfg.bc[2 * d + 1] == FVG_BC_PERIODIC && !(split && (r->peer[0] || r->peer[1]));
        for (int h = 0; h < 2; ++h) a.through[2 * d + h] = a.periodic[d] || r->bc.halo[2 * d + h] == kHaloPeer;
    }
    a.U = Uin;
    a.Rv = r->Rv;
    a.Rvf = r->cfg.precision == FVG_PREC_MIXED && r->dim == 3 ? reinterpret_cast<float*>(r->Rv) : nullptr;
    a.blockmax = bmv;
    a.gate = gate;
    for (int d = 0; d < 3; ++d) a.tiles[d] = r->ntiles_v[d];
    return a;
}

HancockArgs hancock_args(fvg_run* r, const double* Uin, double* out, int mode, double* bm, const int* gate) {
    HancockArgs a{};
    a.m = r->m;
    a.bc = r->bc;
    a.eos = r->eos;
    a.shock_blend = r->cfg.shock_blend;
    a.limiter = r->cfg.limiter;
    a.mode = mode;
    a.U = Uin;
    a.Rv = r->cfg.use_viscous ? r->Rv : nullptr;
    a.out = out;
    a.blockmax = bm;
    a.ctl = r->ctl;
    a.gate = gate;
    for (int d = 0; d < 3; ++d) a.tiles[d] = r->ntiles_h[d];
    return a;
}

cudaError_t launch_hancock(fvg_run* r, const HancockArgs& a) {
    if (r->cfg.riemann == FVG_RIEMANN_LOWMACH)
        return r->full ? launch_hancock_t<kLowMach, true>(r->dim, a, r->nbh, r->stream) : launch_hancock_t<kLowMach, false>(r->dim, a, r->nbh, r->stream);
    return r->full ? launch_hancock_t<kHLLC, true>(r->dim, a, r->nbh, r->stream) : launch_hancock_t<kHLLC, false>(r->dim, a, r->nbh, r->stream);
}

void timer_mark(fvg_run* r, fvg_run::EvTimer& t) {
    if (!r->timing) return;
    if (t.used == t.ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        t.ev.push_back(e);
    }
    cudaEventRecord(t.ev[t.used++], r->stream);
}

// after a stream synchronisation: add up the recorded (start, end) pairs of the first `steps` steps enqueued since the
// last flush (the steps that ran; the gated launches of steps past the end are not counted)
void timer_flush(fvg_run::EvTimer& t, long long steps = -1) {
    const size_t end = (steps >= 0 && (size_t)steps < t.step_start.size()) ? t.step_start[steps] : t.used;
    t.step_start.clear();
    for (size_t k = 0; k + 1 < end; k += 2) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, t.ev[k], t.ev[k + 1]) == cudaSuccess) {
            t.ms += ms;
            t.n += 1;
        }
    }
    t.used = 0;
}

// The immersed body's forced states of Uin (reset = 0: for the residual that follows) or its per-step reset of Uout in
// place (reset = 1: ImmersedBoundary::apply_solid_reset, after each step).
cudaError_t ibm_fill(fvg_run* r, const double* Usrc, double* Uout, int reset, const int* gate) {
    IbmArgs a{};
    a.m = r->m;
    a.eos = r->eos;
    a.slip = r->cfg.use_viscous ? 0 : 1;
    a.ng = r->ng;
    a.nd = r->nd;
    a.ghost = r->d_ghost;
    a.img_cell = r->d_img_cell;
    a.img_w = r->d_img_w;
    a.ratio = r->d_ratio;
    a.gn = r->d_gn;
    a.deep = r->d_deep;
    a.rho_ref = r->cfg.rho_in;
    a.p_ref = r->cfg.p_out;
    a.gvel = r->moving ? r->d_gvel : nullptr;
    a.dvel = r->moving ? r->d_dvel : nullptr;
    a.hydro = r->bc.grav_on && (r->bc.grav[0] != 0.0 || r->bc.grav[1] != 0.0 || r->bc.grav[2] != 0.0);   // set_gravity
    for (int d = 0; d < 3; ++d) a.grav[d] = r->bc.grav[d];
    a.span = r->d_span;
    a.U = Usrc;
    a.forced = r->d_forced;
    a.Uout = Uout;
    a.reset = reset;
    a.gate = gate;
    const int n = r->ng + r->nd;
    const int blocks = n <= 0 ? 1 : ((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184);
    if (r->nvar == 5)
        ibm_fill_kernel<5><<<blocks, 256, 0, r->stream>>>(a);
    else
        ibm_fill_kernel<4><<<blocks, 256, 0, r->stream>>>(a);
    return cudaGetLastError();
}

// The mass-flow inlets' targets of the state a residual is taken of (before the residual's kernels read a ghost).
cudaError_t massflow_targets(fvg_run* r, const double* Uin, const int* gate) {
    if (!r->d_utarget) return cudaSuccess;
    if (r->nvar == 5)
        k_massflow<5><<<6, 1024, 0, r->stream>>>(r->m, r->bc, Uin, r->cfg.rho_in, r->cfg.u_in, r->d_utarget, gate);
    else
        k_massflow<4><<<6, 1024, 0, r->stream>>>(r->m, r->bc, Uin, r->cfg.rho_in, r->cfg.u_in, r->d_utarget, gate);
    return cudaGetLastError();
}

// The viscous residual of Uin into Rv and its per-CTA speed bounds into bmv.
cudaError_t launch_visc(fvg_run* r, const double* Uin, double* bmv, const int* gate, bool timed = true) {
    if (timed) timer_mark(r, r->t_visc);
    const cudaError_t e = r->dim == 2 ? launch_viscous2d(visc_args(r, Uin, bmv, gate), r->nbv, r->stream)
                          : r->cfg.precision == FVG_PREC_MIXED ? mixed_viscous_launch(visc_args(r, Uin, bmv, gate), r->nbv, r->stream)
                                                               : launch_viscous(visc_args(r, Uin, bmv, gate), r->nbv, r->stream);
    if (timed) timer_mark(r, r->t_visc);
    return e;
}

// The residual stage of flux_quadrature = fourth: the face passes of fourth.cuh with the stage's arguments.
template <int DIM, int RIEMANN> cudaError_t fourth_stage_t(fvg_run* r, const StageArgs& sa) {
    constexpr int NV = DIM == 3 ? 5 : 4;
    FourthArgs a = r->fa;
    a.m = sa.m;
    a.bc = sa.bc;
    a.eos = sa.eos;
    a.U = sa.U;
    a.mode = sa.mode;
    a.ca = sa.ca;
    a.cb = sa.cb;
    a.U0 = sa.U0;
    a.out = sa.out;
    a.Rv = sa.Rv;
    a.blockmax = sa.blockmax;
    a.ctl = sa.ctl;
    a.gate = sa.gate;
    auto grid = [](long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); };
    cudaStream_t s = r->stream;
    if (r->cfg.reconstruction == FVG_RECON_WENO5) {
        k4_recon<DIM, NV, 0, true><<<grid(a.nf[0]), 256, 0, s>>>(a);
        k4_recon<DIM, NV, 1, true><<<grid(a.nf[1]), 256, 0, s>>>(a);
        if constexpr (DIM == 3) k4_recon<DIM, NV, 2, true><<<grid(a.nf[2]), 256, 0, s>>>(a);
    } else {
        k4_recon<DIM, NV, 0, false><<<grid(a.nf[0]), 256, 0, s>>>(a);
        k4_recon<DIM, NV, 1, false><<<grid(a.nf[1]), 256, 0, s>>>(a);
        if constexpr (DIM == 3) k4_recon<DIM, NV, 2, false><<<grid(a.nf[2]), 256, 0, s>>>(a);
    }
    k4_point<DIM, NV, 0><<<grid(a.nf[0]), 256, 0, s>>>(a);
    k4_point<DIM, NV, 1><<<grid(a.nf[1]), 256, 0, s>>>(a);
    if constexpr (DIM == 3) k4_point<DIM, NV, 2><<<grid(a.nf[2]), 256, 0, s>>>(a);
    k4_flux<DIM, NV, RIEMANN><<<r->nb, 256, 0, s>>>(a);   // (one CTA per stage tile: the speeds go where the stage kernel's go)
    k4_correct<DIM, NV, RIEMANN, 0><<<grid(a.nf[0]), 256, 0, s>>>(a);
    k4_correct<DIM, NV, RIEMANN, 1><<<grid(a.nf[1]), 256, 0, s>>>(a);
    if constexpr (DIM == 3) k4_correct<DIM, NV, RIEMANN, 2><<<grid(a.nf[2]), 256, 0, s>>>(a);
    k4_balance<DIM, NV><<<grid(r->m.ncells), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fourth_stage(fvg_run* r, const StageArgs& sa) {
    if (r->dim == 3) return r->cfg.riemann == FVG_RIEMANN_LOWMACH ? fourth_stage_t<3, kLowMach>(r, sa) : fourth_stage_t<3, kHLLC>(r, sa);
    return r->cfg.riemann == FVG_RIEMANN_LOWMACH ? fourth_stage_t<2, kLowMach>(r, sa) : fourth_stage_t<2, kHLLC>(r, sa);
}

// The source field's planes of a run: its own planes and, for a part, the ghost planes beyond its interfaces.
void source_planes(const fvg_run* r, int* split, int* first, int* lo, int* hi) {
    *split = r->is_part ? r->split : (r->dim == 3 ? 2 : 1);
    *first = r->is_part ? r->first : 0;
    *lo = r->is_part && r->peer[0] ? r->depth : 0;
    *hi = r->is_part && r->peer[1] ? r->depth : 0;
}

// Before a residual whose stage time is of `kind` (k_stage_values): the stage time, the time-dependent boundary values
// and an unsteady source field.
cudaError_t stage_values(fvg_run* r, int kind, const int* gate) {
    if (!r->tv_on && !r->src_unsteady) return cudaSuccess;
    k_stage_values<<<1, 1, 0, r->stream>>>(r->ctl, gate, kind, r->res_time, r->xa, r->tv_on ? r->d_tv : nullptr);
    if (r->src_unsteady) {
        int split, first, lo, hi;
        source_planes(r, &split, &first, &lo, &hi);
        const long long n = ((split == 2 ? r->m.nz : r->m.ny) + lo + hi) * (split == 2 ? (long long)r->m.nx * r->m.ny : r->m.nx);
        const int blocks = (int)std::min<long long>((n + 127) / 128, 148 * 8);
        if (r->nvar == 5)
            k_source_field<5><<<blocks, 128, 0, r->stream>>>(r->m, r->xa, r->ctl, gate, split, first, lo, hi, r->nsplit, r->d_src + r->goff);
        else
            k_source_field<4><<<blocks, 128, 0, r->stream>>>(r->m, r->xa, r->ctl, gate, split, first, lo, hi, r->nsplit, r->d_src + r->goff);
    }
    return cudaGetLastError();
}

// One residual stage of Uin: the immersed body's forced states, the viscous sweep (viscous runs), then the inviscid
// stage kernel.
cudaError_t residual_stage(fvg_run* r, const double* Uin, const double* U0, double* out, int mode, double ca, double cb, int stage, const int* gate,
                           const unsigned char* fb = nullptr) {
    cudaError_t e;
    if ((e = stage_values(r, r->res_kind >= 0 ? r->res_kind : stage, gate)) != cudaSuccess) return e;
    if (r->ibm && (e = ibm_fill(r, Uin, nullptr, 0, gate)) != cudaSuccess) return e;
    if ((e = massflow_targets(r, Uin, gate)) != cudaSuccess) return e;
    if (r->cfg.use_viscous && (e = launch_visc(r, Uin, r->bmv[stage], gate)) != cudaSuccess) return e;
    timer_mark(r, r->t_stage);
    StageArgs sa = stage_args(r, Uin, U0, out, mode, ca, cb, r->cfg.use_viscous ? r->Rv : nullptr, r->bm[stage], gate);
    sa.fb = fb;
    e = r->fourth ? fourth_stage(r, sa) : r->stage.launch(sa, r->nb, r->stream);
    timer_mark(r, r->t_stage);
    return e;
}

// The sensor's refresh of the gate (a gated run only): at the steps where ctl->steps % sens_every == 0 (ctl null: now).
cudaError_t refresh_gate(fvg_run* r, const double* Uin, const Ctl* ctl) {
    if (!r->sens) return cudaSuccess;
    int per[3];
    for (int d = 0; d < 3; ++d) per[d] = r->cfg.bc[2 * d] == FVG_BC_PERIODIC && r->cfg.bc[2 * d + 1] == FVG_BC_PERIODIC;
    // a part: its split axis does not wrap (beyond an interface lie the neighbour's cells, whose flags are not held here)
    const bool interfaces = r->is_part && (r->peer[0] || r->peer[1]);
    if (interfaces) per[r->split] = 0;
    const int tile[3] = {r->dim == 3 ? Tile<3>::X : Tile<2>::X, r->dim == 3 ? Tile<3>::Y : Tile<2>::Y, r->dim == 3 ? Tile<3>::Z : 1};
    return sensor_refresh(r->m, r->bc, r->eos, r->dim, Uin, r->sens, r->sens_theta, r->sens_radius, per, r->sens_flags, r->sens_flags + (size_t)r->m.plane * r->dim, tile,
                          r->tiles, r->sens_tiles, ctl, r->sens_every, r->sens_count, r->stream, interfaces ? r->split : -1, r->peer[0], r->peer[1]);
}

int axpy_blocks(const fvg_run* r) {
    const long long n = r->m.ncells * r->nvar;
    long long b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? b : 148 * 16);
}

// positivity_fallback: TimeScheme::repair (TimeScheme.cpp:86-90) on the device. Up to kMaxRepairs = 8 times: mark the
// candidate (new cells without density or pressure join the stage's flagged set and raise fb_grew); if one did, `again`
// recomputes the candidate with first-order faces around the set (gated by fb_grew). Then the set is emptied. The
// repeats' wave speeds are not used (the stage's speed is its first residual's).
template <typename F> cudaError_t fb_repair(fvg_run* r, const double* cand, F again) {
    cudaError_t e;
    for (int it = 0; it < 8; ++it) {
        if ((e = cudaMemsetAsync(r->fb_grew, 0, sizeof(int), r->stream))) return e;
        if (r->nvar == 5)
            k_fb_mark<5><<<axpy_blocks(r), 256, 0, r->stream>>>(r->ctl, r->eos, cand, r->m.plane, r->m.ncells, r->fb_flags, r->fb_grew);
        else
            k_fb_mark<4><<<axpy_blocks(r), 256, 0, r->stream>>>(r->ctl, r->eos, cand, r->m.plane, r->m.ncells, r->fb_flags, r->fb_grew);
        if ((e = cudaGetLastError())) return e;
        if ((e = again())) return e;
    }
    return cudaMemsetAsync(r->fb_flags, 0, r->m.ncells, r->stream);
}

// A Runge-Kutta / Euler step with the guard (TimeScheme.cpp:110-290 with guard_): every stage writes its candidate into a
// buffer that is not one of its inputs (Ut, R, Ut), so a repeat recomputes it from the same inputs; the accepted
// candidate is then copied into U. Without repairs the bits are those of the unguarded step.
cudaError_t enqueue_step_fb(fvg_run* r) {
    cudaError_t e;
    Ctl* c = r->ctl;
    const int* act = &c->active;
    const int* rep = r->fb_grew;
    const int nbv = r->cfg.use_viscous ? r->nbv : 0;
    const int ts = r->cfg.time_scheme;
    const long long pl = r->m.plane, n = r->m.ncells;
    const int nv = r->nvar;
    cudaStream_t s = r->stream;
    // stage 1: candidate Ut = U + dt R
    if ((e = residual_stage(r, r->U, nullptr, r->R, kStoreR, 0, 0, 0, act))) return e;
    k_stage1_dt<<<1, 1024, 0, s>>>(c, r->bm[0], r->nb, r->bmv[0], nbv);
    k_axpy<<<axpy_blocks(r), 256, 0, s>>>(c, r->Ut, r->U, r->R, pl, n, nv);
    if ((e = fb_repair(r, r->Ut, [&] {
             cudaError_t e2 = residual_stage(r, r->U, nullptr, r->R, kStoreR, 0, 0, 0, rep, r->fb_flags);
             if (e2) return e2;
             k_axpy_gated<<<axpy_blocks(r), 256, 0, s>>>(rep, c, r->Ut, r->U, r->R, pl, n, nv);
             return cudaGetLastError();
         })))
        return e;
    const double* accepted = r->Ut;
    if (ts == FVG_TS_SSPRK2) {   // stage 2: candidate R = 1/2 U + 1/2 (Ut + dt R(Ut))
        if ((e = residual_stage(r, r->Ut, r->U, r->R, kCombine, 0.5, 0.5, 1, act))) return e;
        k_stage_max<<<1, 1024, 0, s>>>(c, act, 1, r->bm[1], r->nb, r->bmv[1], nbv);
        if ((e = fb_repair(r, r->R, [&] { return residual_stage(r, r->Ut, r->U, r->R, kCombine, 0.5, 0.5, 1, rep, r->fb_flags); }))) return e;
        accepted = r->R;
    } else if (ts == FVG_TS_SSPRK3) {   // stage 2 into R, stage 3 into Ut
        if ((e = residual_stage(r, r->Ut, r->U, r->R, kCombine, 0.75, 0.25, 1, act))) return e;
        k_stage_max<<<1, 1024, 0, s>>>(c, act, 1, r->bm[1], r->nb, r->bmv[1], nbv);
        if ((e = fb_repair(r, r->R, [&] { return residual_stage(r, r->Ut, r->U, r->R, kCombine, 0.75, 0.25, 1, rep, r->fb_flags); }))) return e;
        if ((e = residual_stage(r, r->R, r->U, r->Ut, kCombine, 1.0 / 3.0, 2.0 / 3.0, 2, act))) return e;
        k_stage_max<<<1, 1024, 0, s>>>(c, act, 2, r->bm[2], r->nb, r->bmv[2], nbv);
        if ((e = fb_repair(r, r->Ut, [&] { return residual_stage(r, r->R, r->U, r->Ut, kCombine, 1.0 / 3.0, 2.0 / 3.0, 2, rep, r->fb_flags); })))
            return e;
        accepted = r->Ut;
    }
    k_copy_planes<<<axpy_blocks(r), 256, 0, s>>>(c, r->U, accepted, pl, n, nv);
    if (r->ibm && (e = ibm_fill(r, r->U, r->U, 1, act))) return e;
    k_end_rk<<<1, 1, 0, s>>>(c, ts == FVG_TS_EULER ? 1 : (ts == FVG_TS_SSPRK2 ? 2 : 3));
    return cudaGetLastError();
}

// The launches of one time step on the run's stream (no host synchronisation). refresh = false leaves out the sensor's
// refresh (a graph of sens_every steps keeps it in its first step only).
cudaError_t enqueue_step(fvg_run* r, bool refresh = true) {
    if (r->fb_flags) return enqueue_step_fb(r);
    cudaError_t e;
    Ctl* c = r->ctl;
    const int* act = &c->active;
    const int nbv = r->cfg.use_viscous ? r->nbv : 0;
    const int ts = r->cfg.time_scheme;
    if (ts == FVG_TS_HANCOCK) {
        double* Uin = r->Ucur();
        double* Uout = r->cur ? r->U : r->Ut;
        k_hancock_begin<<<1, 1, 0, r->stream>>>(c);
        // the seed (first step only; untimed): one plain residual for the speed, its viscous bound included
        if ((e = stage_values(r, 0, &c->seed))) return e;
        if (r->ibm && (e = ibm_fill(r, Uin, nullptr, 0, &c->seed))) return e;
        if ((e = massflow_targets(r, Uin, &c->seed))) return e;
        if (r->cfg.use_viscous && (e = launch_visc(r, Uin, r->bmv[1], &c->seed, false))) return e;
        if ((e = r->stage.launch(stage_args(r, Uin, nullptr, r->R, kStoreR, 0, 0, r->cfg.use_viscous ? r->Rv : nullptr, r->bm_seed, &c->seed), r->nb,
                                 r->stream)))
            return e;
        k_hancock_seed<<<1, 1024, 0, r->stream>>>(c, r->bm_seed, r->nb, r->bmv[1], nbv);
        k_hancock_dt<<<1, 1, 0, r->stream>>>(c);
        if ((e = stage_values(r, 2, act))) return e;   // t + dt / 2: the sources centred in the step
        if (r->ibm && (e = ibm_fill(r, Uin, nullptr, 0, act))) return e;
        if ((e = massflow_targets(r, Uin, act))) return e;
        if (r->cfg.use_viscous && (e = launch_visc(r, Uin, r->bmv[0], act))) return e;
        timer_mark(r, r->t_stage);
        e = launch_hancock(r, hancock_args(r, Uin, Uout, kAxpy, r->bm[0], act));
        timer_mark(r, r->t_stage);
        if (e) return e;
        if (r->ibm && (e = ibm_fill(r, Uout, Uout, 1, act))) return e;
        k_hancock_end<<<1, 1024, 0, r->stream>>>(c, r->bm[0], r->nbh, r->bmv[0], nbv);
        r->cur ^= 1;
        return cudaGetLastError();
    }
    if (refresh && (e = refresh_gate(r, r->U, c))) return e;
    if ((e = residual_stage(r, r->U, nullptr, r->R, kStoreR, 0, 0, 0, act))) return e;
    k_stage1_dt<<<1, 1024, 0, r->stream>>>(c, r->bm[0], r->nb, r->bmv[0], nbv);
    if (r->dynamic) {   // a body driven by the flow: the loads of this first stage, about the pivot of the step
        const double vol = r->dim == 3 ? r->m.dx * r->m.dy * r->m.dz : r->m.dx * r->m.dy;
        k_body_loads<<<1, 32, 0, r->stream>>>(act, r->R, r->U, r->m.plane, r->d_solid, r->nsolid, vol, r->m.nx, r->m.ny, r->m.dx, r->m.dy, r->m.dz,
                                              r->dim == 3, r->cfg.ibm_cx + r->body.x, r->cfg.ibm_cy + r->body.y, r->cfg.ibm_cz + r->body.z,
                                              r->bc.grav_on, r->bc.grav[0], r->bc.grav[1], r->bc.grav[2], r->d_bload);
    }
    if (ts == FVG_TS_EULER) {
        k_axpy<<<axpy_blocks(r), 256, 0, r->stream>>>(c, r->U, r->U, r->R, r->m.plane, r->m.ncells, r->nvar);
        if (r->ibm && (e = ibm_fill(r, r->U, r->U, 1, act))) return e;
        k_end_rk<<<1, 1, 0, r->stream>>>(c, 1);
        return cudaGetLastError();
    }
    k_axpy<<<axpy_blocks(r), 256, 0, r->stream>>>(c, r->Ut, r->U, r->R, r->m.plane, r->m.ncells, r->nvar);
    if (ts == FVG_TS_SSPRK2) {
        if ((e = residual_stage(r, r->Ut, r->U, r->U, kCombine, 0.5, 0.5, 1, act))) return e;
        k_stage_max<<<1, 1024, 0, r->stream>>>(c, act, 1, r->bm[1], r->nb, r->bmv[1], nbv);
        if (r->ibm && (e = ibm_fill(r, r->U, r->U, 1, act))) return e;
        k_end_rk<<<1, 1, 0, r->stream>>>(c, 2);
        return cudaGetLastError();
    }
    if ((e = residual_stage(r, r->Ut, r->U, r->R, kCombine, 0.75, 0.25, 1, act))) return e;
    k_stage_max<<<1, 1024, 0, r->stream>>>(c, act, 1, r->bm[1], r->nb, r->bmv[1], nbv);
    if ((e = residual_stage(r, r->R, r->U, r->U, kCombine, 1.0 / 3.0, 2.0 / 3.0, 2, act))) return e;
    k_stage_max<<<1, 1024, 0, r->stream>>>(c, act, 2, r->bm[2], r->nb, r->bmv[2], nbv);
    if (r->ibm && (e = ibm_fill(r, r->U, r->U, 1, act))) return e;
    k_end_rk<<<1, 1, 0, r->stream>>>(c, 3);
    return cudaGetLastError();
}

// ---- parts of a slab-decomposed mesh: a step in phases separated by the hosts' communication
int xblocks(const fvg_run* r) {
    const long long b = (r->xcount + 255) / 256;
    return (int)(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}
cudaError_t part_pack(fvg_run* r, const double* U) {
    k_part_pack<<<xblocks(r), 256, 0, r->stream>>>(U, r->m.plane, r->area, r->depth, r->count, r->nvar, r->xbuf, r->xbuf + r->xcount, r->peer[0],
                                                  r->peer[1]);
    return cudaGetLastError();
}
cudaError_t part_unpack(fvg_run* r, double* U) {
    k_part_unpack<<<xblocks(r), 256, 0, r->stream>>>(U, r->m.plane, r->area, r->depth, r->count, r->nvar, r->xbuf + 2 * r->xcount,
                                                    r->xbuf + 3 * r->xcount, r->peer[0], r->peer[1]);
    return cudaGetLastError();
}
cudaError_t part_local(fvg_run* r, const int* gate, const double* bm, int nb, const double* bmv, int nbv, int slot) {
    k_part_local<<<1, 1024, 0, r->stream>>>(gate, bm, nb, bmv, nbv, r->xred + slot);
    return cudaGetLastError();
}

// Phase `phase` of a step of a part (the launches of enqueue_step, cut where a stage needs its neighbours' planes or
// the speed of every part). *comm: 0 the step is complete; 1 the hosts exchange the send / receive buffers (each part's
// send_lo to its low neighbour's recv_hi, send_hi to its high neighbour's recv_lo); 2 they all-reduce (MAX) the first
// *nred doubles of the reduce buffer; -1 no such phase.
cudaError_t part_phase(fvg_run* r, int phase, int* comm, int* nred) {
    Ctl* c = r->ctl;
    const int* act = &c->active;
    const int nbv = r->cfg.use_viscous ? r->nbv : 0;
    const int ts = r->cfg.time_scheme;
    cudaStream_t s = r->stream;
    cudaError_t e = cudaSuccess;
    *comm = -1;
    *nred = 0;
    if (ts == FVG_TS_HANCOCK) {
        double* Uin = r->Ucur();
        double* Uout = r->cur ? r->U : r->Ut;
        switch (phase) {
        case 0:   // the state's boundary planes
            e = part_pack(r, Uin);
            *comm = 1;
            break;
        case 1:   // the seed residual (first step only) and its speed
            if ((e = part_unpack(r, Uin))) break;
            k_hancock_begin<<<1, 1, 0, s>>>(c);
            if ((e = stage_values(r, 0, &c->seed))) break;
            if (r->cfg.use_viscous && (e = launch_visc(r, Uin, r->bmv[1], &c->seed, false))) break;
            if ((e = r->stage.launch(stage_args(r, Uin, nullptr, r->R, kStoreR, 0, 0, r->cfg.use_viscous ? r->Rv : nullptr, r->bm_seed, &c->seed), r->nb,
                                     s)))
                break;
            e = part_local(r, &c->seed, r->bm_seed, r->nb, r->bmv[1], nbv, 0);
            *comm = 2;
            *nred = 1;
            break;
        case 2:   // dt from the lagged speed, the predictor and update, the speed
            k_part_seed<<<1, 1, 0, s>>>(c, r->xred);
            k_hancock_dt<<<1, 1, 0, s>>>(c);
            if ((e = stage_values(r, 2, act))) break;
            if (r->cfg.use_viscous && (e = launch_visc(r, Uin, r->bmv[0], act))) break;
            timer_mark(r, r->t_stage);
            e = launch_hancock(r, hancock_args(r, Uin, Uout, kAxpy, r->bm[0], act));
            timer_mark(r, r->t_stage);
            if (e) break;
            e = part_local(r, act, r->bm[0], r->nbh, r->bmv[0], nbv, 0);
            *comm = 2;
            *nred = 1;
            break;
        case 3:
            k_part_hancock_end<<<1, 1, 0, s>>>(c, r->xred);
            r->cur ^= 1;
            e = cudaGetLastError();
            *comm = 0;
            break;
        default: break;
        }
        return e;
    }
    switch (phase) {
    case 0:
        e = part_pack(r, r->U);
        *comm = 1;
        break;
    case 1:   // the sensor's refresh on its steps (the state's ghost planes now current), stage 1 and its speed
        if ((e = part_unpack(r, r->U))) break;
        if (r->sens && (e = refresh_gate(r, r->U, c))) break;
        if ((e = residual_stage(r, r->U, nullptr, r->R, kStoreR, 0, 0, 0, act))) break;
        e = part_local(r, act, r->bm[0], r->nb, r->bmv[0], nbv, 0);
        *comm = 2;
        *nred = 1;
        break;
    case 2:   // dt; Euler: the update and the end; else the first stage state and its planes
        k_part_dt<<<1, 1, 0, s>>>(c, r->xred);
        if (ts == FVG_TS_EULER) {
            k_axpy<<<axpy_blocks(r), 256, 0, s>>>(c, r->U, r->U, r->R, r->m.plane, r->m.ncells, r->nvar);
            k_end_rk<<<1, 1, 0, s>>>(c, 1);
            e = cudaGetLastError();
            *comm = 0;
            break;
        }
        k_axpy<<<axpy_blocks(r), 256, 0, s>>>(c, r->Ut, r->U, r->R, r->m.plane, r->m.ncells, r->nvar);
        if ((e = cudaGetLastError())) break;
        e = part_pack(r, r->Ut);
        *comm = 1;
        break;
    case 3:   // stage 2
        if ((e = part_unpack(r, r->Ut))) break;
        if (ts == FVG_TS_SSPRK2) {
            if ((e = residual_stage(r, r->Ut, r->U, r->U, kCombine, 0.5, 0.5, 1, act))) break;
            e = part_local(r, act, r->bm[1], r->nb, r->bmv[1], nbv, 0);
            *comm = 2;
            *nred = 1;
            break;
        }
        if ((e = residual_stage(r, r->Ut, r->U, r->R, kCombine, 0.75, 0.25, 1, act))) break;
        if ((e = part_local(r, act, r->bm[1], r->nb, r->bmv[1], nbv, 0))) break;
        e = part_pack(r, r->R);
        *comm = 1;
        break;
    case 4:
        if (ts == FVG_TS_SSPRK2) {
            k_part_stages<<<1, 1, 0, s>>>(c, r->xred, 1, 1);
            k_end_rk<<<1, 1, 0, s>>>(c, 2);
            e = cudaGetLastError();
            *comm = 0;
            break;
        }
        if ((e = part_unpack(r, r->R))) break;   // stage 3
        if ((e = residual_stage(r, r->R, r->U, r->U, kCombine, 1.0 / 3.0, 2.0 / 3.0, 2, act))) break;
        e = part_local(r, act, r->bm[2], r->nb, r->bmv[2], nbv, 1);
        *comm = 2;
        *nred = 2;
        break;
    case 5:
        if (ts != FVG_TS_SSPRK3) break;
        k_part_stages<<<1, 1, 0, s>>>(c, r->xred, 1, 2);
        k_end_rk<<<1, 1, 0, s>>>(c, 3);
        e = cudaGetLastError();
        *comm = 0;
        break;
    default: break;
    }
    return e;
}

int read_ctl(fvg_run* run, Ctl* h) {
    CK(cudaMemcpyAsync(h, run->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, run->stream));
    CK(cudaStreamSynchronize(run->stream));
    return FVG_OK;
}

}   // namespace

// configuration checks shared with the batched runs (batch.cu)
std::string fvg::config_error(const fvg_config& c) { return validate(c); }
bool fvg::config_has_expressions(const fvg_config& c) { return has_expressions(c); }
void fvg::config_halo_kinds(const fvg_config& c, int depth, int kinds[6]) { halo_kinds(c, depth, kinds); }
std::string* fvg::create_error_slot() { return &g_create_error; }
bool fvg::run_view(fvg_run* run, RunView* v) {
    if (!run || !v) return false;
    v->m = run->m;
    v->bc = run->bc;
    v->eos = run->eos;
    v->U = run->Ucur();
    v->stream = run->stream;
    v->dim = run->dim;
    v->nvar = run->nvar;
    v->device = run->cfg.device;
    v->weno_eps = run->cfg.weno_epsilon;
    return true;
}

namespace {
int create_run(const fvg_config* cfg, int nparts, int part, bool as_part, fvg_run** out);
}

// ------------------------------------------------------------------------------------------------ C ABI
extern "C" {

int fvg_abi_version(void) { return FVG_ABI_VERSION; }
const char* fvg_create_error(void) { return g_create_error.c_str(); }
const char* fvg_last_error(const fvg_run* run) { return run ? run->err.c_str() : "null run"; }

int fvg_create(const fvg_config* cfg, fvg_run** out) { return create_run(cfg, 1, 0, false, out); }

int fvg_create_part(const fvg_config* cfg, int nparts, int part, fvg_run** out) {
    if (nparts < 1 || part < 0 || part >= nparts) {
        g_create_error = "part must be in 0 .. nparts - 1";
        return FVG_ERR_ARGUMENT;
    }
    return create_run(cfg, nparts, part, true, out);
}

}   // extern "C"

namespace {

// The case-file expressions of a run (Simulation::setup and load_boundary_functions, cpp/src/Simulation.cpp:118-168,
// 372-412): compiles the source terms (when one is not a whole number equal to 0) and the boundary values given as
// expressions of t or time tables, replaces u_in, v_in, rho_in, p_out by their values at t = 0, and notes which vary.
// Throws std::exception with the reference's message for what it refuses.
void compile_expressions(fvg_run* run, const fvg_config& whole, expr::Program& p) {
    for (int i = 0; i < whole.nparams; ++i) p.bind(whole.param_names[i] ? whole.param_names[i] : "", whole.param_values[i]);
    p.bind("Lx", whole.Lx);   // the mesh is authoritative for the domain (CaseFile.cpp:323-329)
    p.bind("Ly", whole.Ly);
    p.bind("Lz", whole.Lz);
    p.bind("nx", whole.nx);
    p.bind("ny", whole.ny);
    p.bind("nz", whole.nz);
    static const char* const skeys[5] = {"source_rho", "source_mx", "source_my", "source_E", "source_mz"};
    bool use = false;
    for (int q = 0; q < 5; ++q) {
        const char* v = whole.source[q] ? whole.source[q] : "0";
        char* end = nullptr;
        const double d = std::strtod(v, &end);
        if (!(end && *end == '\0' && d == 0.0)) use = true;
    }
    for (int q = 0; q < 5; ++q) run->xa.src[q] = -1;
    if (use) {
        for (int q = 0; q < 5; ++q) {
            run->xa.src[q] = p.add(whole.source[q] ? whole.source[q] : "0", skeys[q]);
            if (p.reads(run->xa.src[q], expr::kVarT)) run->src_unsteady = true;
        }
        run->src_on = true;
        double c0 = 0.0;
        if (whole.nz <= 1 && !(p.constant(run->xa.src[4], &c0) && c0 == 0.0))
            throw std::invalid_argument("source_mz must be 0 on a 2-D mesh (rho w is held at 0 there)");
    }
    static const char* const bkeys[4] = {"u_in", "v_in", "rho_in", "p_out"};
    double* vals[4] = {&run->cfg.u_in, &run->cfg.v_in, &run->cfg.rho_in, &run->cfg.p_out};
    bool any = false;
    for (int k = 0; k < 4; ++k) {
        run->xa.bnd[k] = -1;
        const char* ex = whole.boundary_expr[k];
        const bool has_ex = ex && *ex;
        char* end = nullptr;
        const double num = has_ex ? std::strtod(ex, &end) : 0.0;
        const bool numeric = has_ex && end != ex && *end == '\0';
        const std::string key = bkeys[k];
        int entry = -1;
        if (whole.boundary_table[k] && whole.boundary_table_rows[k] > 0) {
            if (has_ex && !numeric) throw std::invalid_argument(key + " expression and " + key + "_table cannot both be set");
            entry = p.add_table(whole.boundary_table[k], whole.boundary_table_rows[k], key + "_table");
        } else if (has_ex) {
            if (numeric) *vals[k] = num;
            else entry = p.add(ex, key);
        }
        if (entry < 0) continue;
        any = true;
        const double v0 = p.eval(entry, 0.0, 0.0, 0.0, 0.0);
        if (!std::isfinite(v0)) throw std::runtime_error(key + ": time expression evaluated to a non-finite value");
        *vals[k] = v0;
        if (p.reads(entry, expr::kVarT)) {
            run->xa.bnd[k] = entry;
            run->tv_on = true;
        }
    }
    if (any && (!(run->cfg.rho_in > 0.0) || !(run->cfg.p_out > 0.0)))
        throw std::invalid_argument("time-dependent rho_in and p_out must be positive at t=0");
}

// The programs on the device, the boundary values' array and the source field (a steady one evaluated here on the
// host, with the C library's functions as the reference evaluates it: its bits; an unsteady one is evaluated on the
// device before every residual).
int upload_expressions(fvg_run* run, const expr::Program& p) {
    if (!run->src_on && !run->tv_on) return FVG_OK;
    if (cudaMalloc(&run->d_code, sizeof(expr::Op) * p.code.size()) != cudaSuccess ||
        cudaMalloc(&run->d_pool, sizeof(double) * (p.pool.size() + 1)) != cudaSuccess || cudaMalloc(&run->d_tv, sizeof(double) * 4) != cudaSuccess)
        return fail(run, FVG_ERR_CUDA, "device allocation failed");
    const double tv0[4] = {run->cfg.u_in, run->cfg.v_in, run->cfg.rho_in, run->cfg.p_out};
    if (cudaMemcpy(run->d_code, p.code.data(), sizeof(expr::Op) * p.code.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        (!p.pool.empty() && cudaMemcpy(run->d_pool, p.pool.data(), sizeof(double) * p.pool.size(), cudaMemcpyHostToDevice) != cudaSuccess) ||
        cudaMemcpy(run->d_tv, tv0, sizeof(tv0), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(run, FVG_ERR_CUDA, "copy of the expression programs failed");
    run->xa.code = run->d_code;
    run->xa.pool = run->d_pool;
    if (run->tv_on) run->bc.tv = run->d_tv;
    if (!run->src_on) return FVG_OK;
    const size_t sbytes = sizeof(double) * run->m.plane * run->nvar;
    if (cudaMalloc(&run->d_src, sbytes) != cudaSuccess) return fail(run, FVG_ERR_CUDA, "device allocation failed");
    run->bc.src = run->d_src + run->goff;
    if (run->src_unsteady) return cudaMemset(run->d_src, 0, sbytes) == cudaSuccess ? FVG_OK : fail(run, FVG_ERR_CUDA, "cudaMemset failed");
    int split, first, lo, hi;
    source_planes(run, &split, &first, &lo, &hi);
    const Mesh& m = run->m;
    const long long nloc = split == 2 ? m.nz : m.ny, area = split == 2 ? (long long)m.nx * m.ny : m.nx;
    std::vector<double> S((size_t)m.plane * run->nvar, 0.0);
    const long long total = (nloc + lo + hi) * area;
    const int nv = run->nvar;
    auto work = [&](long long from, long long to) {   // the cells of k_source_field, the same coordinates
        for (long long e = from; e < to; ++e) {
            const long long pl = e / area - lo, rem = e % area;
            long long gp = first + pl;
            if (gp < 0) gp += run->nsplit;
            else if (gp >= run->nsplit) gp -= run->nsplit;
            const long long i = split == 2 ? rem % m.nx : rem, j = split == 2 ? rem / m.nx : gp, k = split == 2 ? gp : 0;
            const double xc = ((double)i + 0.5) * m.dx, yc = ((double)j + 0.5) * m.dy, zc = nv == 5 ? ((double)k + 0.5) * m.dz : 0.0;
            const long long cell = run->goff + pl * area + rem;
            for (int q = 0; q < nv; ++q) S[(size_t)q * m.plane + cell] = p.eval(run->xa.src[q], xc, yc, zc, 0.0);
        }
    };
    const int nthreads = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (total < (1 << 16) || nthreads == 1) {
        work(0, total);
    } else {
        std::vector<std::thread> pool;
        for (int w = 0; w < nthreads; ++w) pool.emplace_back(work, total * w / nthreads, total * (w + 1) / nthreads);
        for (std::thread& t : pool) t.join();
    }
    if (cudaMemcpy(run->d_src, S.data(), sbytes, cudaMemcpyHostToDevice) != cudaSuccess) return fail(run, FVG_ERR_CUDA, "copy of the source field failed");
    return FVG_OK;
}

// ImmersedBoundary::body_velocity (cpp/src/Physics.cpp:1128-1139): the velocity of the rigid body at (x, y, z), with the
// velocities of the pose and the pivot where the geometry was built.
void body_velocity(const fvg_run* r, double x, double y, double z, double v[3]) {
    const fvg_run::Pose& p = r->pose;
    const double px = r->cfg.ibm_cx + r->built.x, py = r->cfg.ibm_cy + r->built.y;
    v[0] = p.u - p.omega * (y - py);
    v[1] = p.v + p.omega * (x - px);
    v[2] = p.w;
    if (p.omega_x != 0.0 || p.omega_y != 0.0) {
        const double pz = r->cfg.ibm_cz + r->built.z, rx = x - px, ry = y - py, rz = z - pz;
        v[0] += p.omega_y * rz;
        v[1] -= p.omega_x * rz;
        v[2] += p.omega_x * ry - p.omega_y * rx;
    }
}

// The wall velocity of every ghost (at its wall point) and the velocity of every deep cell (at its centre) of a moving
// body, from the current pose (refresh_wall_velocity; the deep cells' of fill_ghosts_part).
int upload_velocities(fvg_run* r) {
    const IbmTable& t = r->tab;
    const int ng = (int)t.ghost.size(), nd = (int)t.deep.size();
    std::vector<double> gv(3 * (size_t)ng + 3), dv(3 * (size_t)nd + 3);
    for (int k = 0; k < ng; ++k) body_velocity(r, t.gwx[k], t.gwy[k], r->dim == 3 ? t.gwz[k] : 0.0, &gv[3 * k]);
    const double dx = r->m.dx, dy = r->m.dy, dz = r->m.dz;
    for (int k = 0; k < nd; ++k) {
        const int c = t.deep[k], i = c % r->m.nx, j = (c / r->m.nx) % r->m.ny, kk = c / (r->m.nx * r->m.ny);
        body_velocity(r, (i + 0.5) * dx + 0.0, (j + 0.5) * dy + 0.0, r->dim == 3 ? (kk + 0.5) * dz + 0.0 : 0.0, &dv[3 * k]);
    }
    if (cudaMemcpy(r->d_gvel, gv.data(), sizeof(double) * gv.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(r->d_dvel, dv.data(), sizeof(double) * dv.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(r, FVG_ERR_CUDA, "copy of the wall velocities failed");
    return FVG_OK;
}

// The immersed body's tables (run->tab) on the device: the mask, the forced-state slots, the ghost and deep cells with
// their image points, the solid cells of the loads and, for a moving body, the velocities. The arrays of an earlier
// geometry are replaced.
int upload_ibm(fvg_run* run) {
    for (void** p : {(void**)&run->d_slot, (void**)&run->d_forced, (void**)&run->d_ghost, (void**)&run->d_img_cell, (void**)&run->d_img_w,
                     (void**)&run->d_ratio, (void**)&run->d_gn, (void**)&run->d_deep, (void**)&run->d_solid, (void**)&run->d_gvel,
                     (void**)&run->d_dvel, (void**)&run->d_span})
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
    const IbmTable& t = run->tab;
    run->ng = (int)t.ghost.size();
    run->nd = (int)t.deep.size();
    std::vector<int> slot(run->m.ncells, -1);
    for (int k = 0; k < run->ng; ++k) slot[t.ghost[k]] = k;
    for (int k = 0; k < run->nd; ++k) slot[t.deep[k]] = run->ng + k;
    std::vector<double> gn(3 * (size_t)run->ng);
    for (int k = 0; k < run->ng; ++k) {
        gn[3 * k] = t.gnx[k];
        gn[3 * k + 1] = t.gny[k];
        gn[3 * k + 2] = t.gnz[k];
    }
    const size_t ns = (size_t)(run->ng + run->nd) + 1, ng1 = (size_t)run->ng + 1, nd1 = (size_t)run->nd + 1;
    bool ok = (run->d_mask || cudaMalloc(&run->d_mask, run->m.ncells) == cudaSuccess) &&
              cudaMalloc(&run->d_slot, sizeof(int) * run->m.ncells) == cudaSuccess && cudaMalloc(&run->d_forced, sizeof(double) * 5 * ns) == cudaSuccess &&
              cudaMalloc(&run->d_ghost, sizeof(int) * ng1) == cudaSuccess && cudaMalloc(&run->d_img_cell, sizeof(int) * 8 * ng1) == cudaSuccess &&
              cudaMalloc(&run->d_img_w, sizeof(double) * 8 * ng1) == cudaSuccess && cudaMalloc(&run->d_ratio, sizeof(double) * ng1) == cudaSuccess &&
              cudaMalloc(&run->d_gn, sizeof(double) * 3 * ng1) == cudaSuccess && cudaMalloc(&run->d_deep, sizeof(int) * nd1) == cudaSuccess &&
              cudaMalloc(&run->d_span, sizeof(double) * ng1) == cudaSuccess &&
              (!run->moving || (cudaMalloc(&run->d_gvel, sizeof(double) * 3 * ng1) == cudaSuccess &&
                                cudaMalloc(&run->d_dvel, sizeof(double) * 3 * nd1) == cudaSuccess));
    ok = ok && cudaMemcpy(run->d_mask, t.mask.data(), run->m.ncells, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(run->d_slot, slot.data(), sizeof(int) * run->m.ncells, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok && run->ng > 0)
        ok = cudaMemcpy(run->d_ghost, t.ghost.data(), sizeof(int) * run->ng, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(run->d_img_cell, t.img_cell.data(), sizeof(int) * 8 * run->ng, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(run->d_img_w, t.img_w.data(), sizeof(double) * 8 * run->ng, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(run->d_ratio, t.ratio.data(), sizeof(double) * run->ng, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(run->d_gn, gn.data(), sizeof(double) * 3 * run->ng, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(run->d_span, t.span.data(), sizeof(double) * run->ng, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok && run->nd > 0) ok = cudaMemcpy(run->d_deep, t.deep.data(), sizeof(int) * run->nd, cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) return fail(run, FVG_ERR_CUDA, "device allocation of the immersed body's tables failed");
    std::vector<int> solid_cells;
    for (long long c = 0; c < run->m.ncells; ++c)
        if (t.mask[c]) solid_cells.push_back((int)c);
    run->nsolid = (int)solid_cells.size();
    if (cudaMalloc(&run->d_solid, sizeof(int) * (solid_cells.size() + 1)) != cudaSuccess ||
        (!run->d_loads && cudaMalloc(&run->d_loads, sizeof(double) * 3) != cudaSuccess) ||
        (run->nsolid > 0 && cudaMemcpy(run->d_solid, solid_cells.data(), sizeof(int) * run->nsolid, cudaMemcpyHostToDevice) != cudaSuccess))
        return fail(run, FVG_ERR_CUDA, "device allocation of the immersed body's tables failed");
    run->bc.solid = run->d_mask;
    run->bc.slot = run->d_slot;
    run->bc.forced = run->d_forced;
    return run->moving ? upload_velocities(run) : FVG_OK;
}

// Simulation::prescribed_pose (cpp/src/SimulationRun.cpp:193-214) at time t.
fvg_run::Pose prescribed_pose(const fvg_config& c, double t) {
    fvg_run::Pose p;
    p.x = c.ibm_vx * t;
    p.y = c.ibm_vy * t;
    p.z = c.ibm_vz * t;
    p.w = c.ibm_vz;
    p.angle = c.ibm_omega * t;
    p.u = c.ibm_vx;
    p.v = c.ibm_vy;
    p.omega = c.ibm_omega;
    p.omega_x = c.ibm_omega_x;
    p.omega_y = c.ibm_omega_y;
    if (c.ibm_omega_from > 0.0 || c.ibm_omega_until > 0.0) {   // the rotation runs between two times, the angle held outside
        const double t_off = c.ibm_omega_until > 0.0 ? c.ibm_omega_until : t;
        p.angle = c.ibm_omega * (vmin(vmax(t, c.ibm_omega_from), vmax(t_off, c.ibm_omega_from)) - c.ibm_omega_from);
        const bool on = t >= c.ibm_omega_from && (c.ibm_omega_until <= 0.0 || t < c.ibm_omega_until);
        p.omega = on ? c.ibm_omega : 0.0;
        p.omega_x = on ? c.ibm_omega_x : 0.0;
        p.omega_y = on ? c.ibm_omega_y : 0.0;
    }
    return p;
}

// Simulation::body_pose (SimulationRun.cpp:216-230): the prescribed pose, or the state of a body driven by the flow.
fvg_run::Pose body_pose(const fvg_run* r, double t) {
    if (!r->dynamic) return prescribed_pose(r->cfg, t);
    fvg_run::Pose p;
    const fvg_run::Body& b = r->body;
    p.x = b.x;
    p.y = b.y;
    p.u = b.u;
    p.v = b.v;
    p.z = b.z;
    p.w = b.w;
    p.angle = b.th;
    p.omega = b.om;
    p.omega_x = b.omx;
    p.omega_y = b.omy;
    return p;
}

// Simulation::coupled_accelerations (SimulationRun.cpp:236-248): the pivot's accelerations and the angular one of a
// body whose centre of mass is off its pivot (gravity: the body force's).
void coupled_accelerations(const fvg_run* r, double acc[3]) {
    const fvg_run::Body& b = r->body;
    const fvg_config& p = r->cfg;
    const double c = std::cos(b.th), s = std::sin(b.th);
    const double rx = r->cm0[0] * c - r->cm0[1] * s, ry = r->cm0[0] * s + r->cm0[1] * c;
    const double fx = b.fx - p.ibm_stiff_x * b.x - p.ibm_damp_x * b.u, fy = b.fy - p.ibm_stiff_y * b.y - p.ibm_damp_y * b.v;
    const double mp = b.mz - p.ibm_stiff_theta * b.th - p.ibm_damp_theta * b.om;
    const double icm = p.ibm_inertia - p.ibm_mass * (rx * rx + ry * ry);
    const double alpha = (mp - (rx * fy - ry * fx)) / icm;
    const double gx = p.use_bodyforce ? p.gx : 0.0, gy = p.use_bodyforce ? p.gy : 0.0;
    acc[0] = fx / p.ibm_mass + gx + alpha * ry + b.om * b.om * rx;
    acc[1] = fy / p.ibm_mass + gy - alpha * rx + b.om * b.om * ry;
    acc[2] = alpha;
}

// Simulation::advance_body (SimulationRun.cpp:250-310): the body's velocities by Adams-Bashforth 2 for a variable step
// (an Euler step after a much shorter one), its displacement and angle by the trapezoid rule, from the loads of the step.
void advance_body(fvg_run* r, double dt) {
    fvg_run::Body& b = r->body;
    const fvg_config& p = r->cfg;
    const bool coupled = p.ibm_cm_x != 0.0 || p.ibm_cm_y != 0.0;
    double acc[3] = {0.0, 0.0, 0.0};
    if (coupled) coupled_accelerations(r, acc);
    if (p.ibm_inertia > 0.0) {
        const bool ab = b.dt > 0.0 && dt <= 2.0 * b.dt;
        const double rr = ab ? dt / b.dt : 0.0;
        const auto advance = [&](double om, double prev, double a) { return ab ? om + dt * ((1.0 + 0.5 * rr) * a - 0.5 * rr * prev) : om + dt * a; };
        const double a = coupled ? acc[2] : (b.mz - p.ibm_stiff_theta * b.th - p.ibm_damp_theta * b.om) / p.ibm_inertia;
        const double om1 = advance(b.om, b.aom, a);
        if (p.nz > 1) {
            const double ax = (b.mx - p.ibm_damp_theta * b.omx) / p.ibm_inertia, ay = (b.my - p.ibm_damp_theta * b.omy) / p.ibm_inertia;
            const double omx1 = advance(b.omx, b.aomx, ax), omy1 = advance(b.omy, b.aomy, ay);
            b.omx = omx1;
            b.omy = omy1;
            b.aomx = ax;
            b.aomy = ay;
        } else {
            b.th += 0.5 * dt * (b.om + om1);
        }
        b.om = om1;
        b.aom = a;
    }
    if (!(p.ibm_mass > 0.0)) {
        b.dt = dt;
        return;
    }
    const double gx = p.use_bodyforce ? p.gx : 0.0, gy = p.use_bodyforce ? p.gy : 0.0;
    const double ax = coupled ? acc[0] : (b.fx - p.ibm_stiff_x * b.x - p.ibm_damp_x * b.u) / p.ibm_mass + gx;
    const double ay = coupled ? acc[1] : (b.fy - p.ibm_stiff_y * b.y - p.ibm_damp_y * b.v) / p.ibm_mass + gy;
    const bool d3 = p.nz > 1;
    const double gz = p.use_bodyforce && d3 ? p.gz : 0.0;
    const double az = d3 ? (b.fz - p.ibm_stiff_z * b.z - p.ibm_damp_z * b.w) / p.ibm_mass + gz : 0.0;
    double u1, v1, w1 = 0.0;
    if (b.dt > 0.0 && dt <= 2.0 * b.dt) {
        const double rr = dt / b.dt;
        u1 = b.u + dt * ((1.0 + 0.5 * rr) * ax - 0.5 * rr * b.ax);
        v1 = b.v + dt * ((1.0 + 0.5 * rr) * ay - 0.5 * rr * b.ay);
        if (d3) w1 = b.w + dt * ((1.0 + 0.5 * rr) * az - 0.5 * rr * b.az);
    } else {
        u1 = b.u + dt * ax;
        v1 = b.v + dt * ay;
        if (d3) w1 = b.w + dt * az;
    }
    b.x += 0.5 * dt * (b.u + u1);
    b.y += 0.5 * dt * (b.v + v1);
    b.u = u1;
    b.v = v1;
    b.ax = ax;
    b.ay = ay;
    if (d3) {
        b.z += 0.5 * dt * (b.w + w1);
        b.w = w1;
        b.az = az;
    }
    b.dt = dt;
}

// The body's geometry at a pose (ImmersedBoundary::place_geometry and build_ghosts, Physics.cpp:1204-1212 and 1310-1334):
// the shape moved by the pose's displacement (a section also turned about its pivot by the pose's angle), its mask and
// ghost table built on the host into tb.
int geometry_at(fvg_run* r, const fvg_run::Pose& pose, IbmGeom& g, IbmTable& tb) {
    g = ibm_geom(r->cfg, r->cfg.ibm_cx + pose.x, r->cfg.ibm_cy + pose.y, r->cfg.ibm_cz + pose.z);
    if (r->cfg.ibm_shape == 2) {   // the section turned about the pivot by the pose's angle and moved by its displacement
        const double ca = std::cos(pose.angle), sa = std::sin(pose.angle), px = r->cfg.ibm_cx, py = r->cfg.ibm_cy;
        std::vector<double> pts(r->ref_poly.size());
        for (size_t q = 0; q < pts.size() / 2; ++q) {
            const double rx = r->ref_poly[2 * q] - px, ry = r->ref_poly[2 * q + 1] - py;
            pts[2 * q] = px + pose.x + ca * rx - sa * ry;
            pts[2 * q + 1] = py + pose.y + sa * rx + ca * ry;
        }
        g.set_polygon(std::move(pts));
    }
    const std::string msg = build_ibm_geom(g, tb);
    if (!msg.empty()) return fail(r, FVG_ERR_CONFIG, msg);
    return FVG_OK;
}

// The body at the start of a step at time t (place_body and ImmersedBoundary::move_to, SimulationRun.cpp:379-384 and
// Physics.cpp:1310-1334): the geometry follows the pose in steps of a quarter cell (then the ghost table is built again
// and the cells the body left take the wall layer's state, fill_fresh); in between only the wall velocities change.
int place_body(fvg_run* r, double t) {
    const fvg_run::Pose pose = body_pose(r, t);
    const double h = r->dim == 3 ? vmin(vmin(r->m.dx, r->m.dy), r->m.dz) : vmin(r->m.dx, r->m.dy);
    const bool poly = r->cfg.ibm_shape == 2;
    const double shift = vmax(vmax(vmax(fabs(pose.x - r->built.x), fabs(pose.y - r->built.y)), fabs(pose.z - r->built.z)),
                              poly ? fabs(pose.angle - r->built.angle) * r->reach : 0.0);
    r->pose = pose;
    if (shift <= 0.25 * h) return upload_velocities(r);
    const std::vector<unsigned char> old_mask = r->tab.mask;
    r->built = pose;
    IbmGeom g;
    IbmTable tb;
    if (const int rc = geometry_at(r, pose, g, tb)) return rc;
    std::vector<int> cells;   // fresh: solid before, fluid now
    for (size_t c = 0; c < tb.mask.size(); ++c)
        if (old_mask[c] && !tb.mask[c]) cells.push_back((int)c);
    FreshTable f;
    build_fresh(g, tb.mask, cells, [&](double x, double y, double z, double* v) { body_velocity(r, x, y, z, v); }, f);
    r->tab = std::move(tb);
    if (cudaStreamSynchronize(r->stream) != cudaSuccess) return fail(r, FVG_ERR_CUDA, "synchronisation failed");
    if (const int rc = upload_ibm(r)) return rc;
    const int n = (int)f.cell.size();
    if (n == 0) return FVG_OK;
    int *dc = nullptr, *di = nullptr;
    double *dw = nullptr, *dr = nullptr, *dv = nullptr;
    bool ok = cudaMalloc(&dc, sizeof(int) * n) == cudaSuccess && cudaMalloc(&di, sizeof(int) * 8 * n) == cudaSuccess &&
              cudaMalloc(&dw, sizeof(double) * 8 * n) == cudaSuccess && cudaMalloc(&dr, sizeof(double) * n) == cudaSuccess &&
              cudaMalloc(&dv, sizeof(double) * 3 * n) == cudaSuccess;
    ok = ok && cudaMemcpy(dc, f.cell.data(), sizeof(int) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(di, f.img_cell.data(), sizeof(int) * 8 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(dw, f.img_w.data(), sizeof(double) * 8 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(dr, f.ratio.data(), sizeof(double) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(dv, f.wvel.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) {
        FreshArgs a{};
        a.m = r->m;
        a.eos = r->eos;
        a.n = n;
        a.cell = dc;
        a.img_cell = di;
        a.img_w = dw;
        a.ratio = dr;
        a.wvel = dv;
        a.U = r->Ucur();
        const int blocks = (n + 255) / 256;
        if (r->nvar == 5)
            fresh_fill_kernel<5><<<blocks, 256, 0, r->stream>>>(a);
        else
            fresh_fill_kernel<4><<<blocks, 256, 0, r->stream>>>(a);
        ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(r->stream) == cudaSuccess;
    }
    for (void* p : {(void*)dc, (void*)di, (void*)dw, (void*)dr, (void*)dv})
        if (p) cudaFree(p);
    return ok ? FVG_OK : fail(r, FVG_ERR_CUDA, "the fill of the cells the body left failed");
}

// fvg_create, and part `part` of `nparts` slabs of the mesh along its slowest axis (nparts = 1 with part mode off: a
// whole run). A part holds planes first .. first + count - 1 of the split axis (the first nsplit % nparts parts one
// plane more), with `depth` ghost planes on each side; the mesh spacing, the step length and every other parameter are
// the whole mesh's.
int create_run(const fvg_config* cfg, int nparts, int part, bool as_part, fvg_run** out) {
    if (!cfg || !out) {
        g_create_error = "null argument";
        return FVG_ERR_ARGUMENT;
    }
    *out = nullptr;
    const std::string v = validate(*cfg);
    if (!v.empty()) {
        g_create_error = v;
        return FVG_ERR_CONFIG;
    }
    const bool is_part = as_part;
    const int split = cfg->nz > 1 ? 2 : 1;
    const int nsplit = split == 2 ? cfg->nz : cfg->ny;
    const int depth = cfg->reconstruction == FVG_RECON_WENO5 ? 3 : 2;
    const int count = nsplit / nparts + (part < nsplit % nparts ? 1 : 0);
    const int first = part * (nsplit / nparts) + (part < nsplit % nparts ? part : nsplit % nparts);
    if (is_part) {
        if (cfg->use_ibm) {
            g_create_error = "a part of a decomposed mesh cannot hold an immersed body";
            return FVG_ERR_CONFIG;
        }
        if (count < depth) {
            g_create_error = "each part needs at least " + std::to_string(depth) + " planes along the split axis";
            return FVG_ERR_CONFIG;
        }
        if (cfg->flux_quadrature == 1) {   // Params.cpp:454
            g_create_error = "flux_quadrature = fourth is serial yet (its corrections read faces two cells across a part interface)";
            return FVG_ERR_CONFIG;
        }
        if (cfg->positivity_fallback) {   // the flags of the neighbours' cells would have to be exchanged too
            g_create_error = "a decomposed mesh cannot use positivity_fallback";
            return FVG_ERR_CONFIG;
        }
        for (int s = 0; s < 6; ++s)
            if (cfg->bc[s] == FVG_BC_MASSFLOWINLET) {   // its target is a sequential sum over the whole side
                g_create_error = "a decomposed mesh cannot have a mass-flow inlet";
                return FVG_ERR_CONFIG;
            }
        // a first-order run takes the states of a periodic side's faces through the round trip (a side without a halo);
        // split there, those faces would be a part interface
        if (cfg->reconstruction == FVG_RECON_NONE && cfg->bc[2 * split] == FVG_BC_PERIODIC) {
            g_create_error = "a first-order run cannot be split along a periodic axis";
            return FVG_ERR_CONFIG;
        }
    }
    auto* run = new fvg_run();
    run->cfg = *cfg;
    if (is_part) {
        const bool periodic = cfg->bc[2 * split] == FVG_BC_PERIODIC && cfg->bc[2 * split + 1] == FVG_BC_PERIODIC;
        run->is_part = true;
        run->nparts = nparts;
        run->part = part;
        run->split = split;
        run->first = first;
        run->count = count;
        run->depth = depth;
        run->peer[0] = part > 0 || periodic;
        run->peer[1] = part < nparts - 1 || periodic;
        (split == 2 ? run->cfg.nz : run->cfg.ny) = count;   // the local mesh; the spacing below is the whole mesh's
    }
    const fvg_config& c = run->cfg;
    auto bail = [&](int code) {
        g_create_error = run->err;
        fvg_destroy(run);
        return code;
    };
    run->nsplit = nsplit;
    expr::Program prog;
    try {
        compile_expressions(run, *cfg, prog);
    } catch (const std::exception& ex) {
        run->err = ex.what();
        return bail(FVG_ERR_CONFIG);
    }
    for (int q = 0; q < 5; ++q) run->cfg.source[q] = nullptr;   // (the caller's memory is not kept)
    for (int k = 0; k < 4; ++k) {
        run->cfg.boundary_expr[k] = nullptr;
        run->cfg.boundary_table[k] = nullptr;
        run->cfg.boundary_table_rows[k] = 0;
    }
    run->cfg.param_names = nullptr;
    run->cfg.param_values = nullptr;
    run->cfg.nparams = 0;
    if (cudaSetDevice(c.device) != cudaSuccess) {
        run->err = "cudaSetDevice failed (no CUDA device?)";
        return bail(FVG_ERR_CUDA);
    }
    run->dim = c.nz > 1 ? 3 : 2;
    run->nvar = run->dim == 3 ? 5 : 4;
    Mesh& m = run->m;
    m.nx = c.nx;
    m.ny = c.ny;
    m.nz = c.nz;
    m.ncells = (long long)c.nx * c.ny * c.nz;
    m.plane = (m.ncells + 31) / 32 * 32;
    if (run->is_part) {   // ghost planes before and after the part's own along the split axis
        run->area = split == 2 ? (long long)c.nx * c.ny : (long long)c.nx;
        run->goff = (long long)depth * run->area;
        m.plane = ((long long)(count + 2 * depth) * run->area + 31) / 32 * 32;
        run->xcount = (long long)depth * run->area * (run->dim == 3 ? 5 : 4);
    }
    const fvg_config& g = *cfg;   // the whole mesh
    m.dx = g.Lx / g.nx;   // generate_cartesian_mesh_3d (Core.cpp:20-40)
    m.dy = g.Ly / g.ny;
    m.dz = g.Lz / g.nz;
    if (run->dim == 3) {
        m.area[0] = m.dy * m.dz;
        m.area[1] = m.dx * m.dz;
        m.area[2] = m.dx * m.dy;
        m.inv_cell = 1.0 / (m.dx * m.dy * m.dz);
        run->L = 2.0 / (1.0 / (g.Lx / g.nx) + 1.0 / (g.Ly / g.ny) + 1.0 / (g.Lz / g.nz));
    } else {
        m.area[0] = m.dy;
        m.area[1] = m.dx;
        m.area[2] = 0.0;
        m.inv_cell = 1.0 / (m.dx * m.dy);
        run->L = vmin(g.Lx / g.nx, g.Ly / g.ny);
    }
    run->eos.type = c.eos_type;
    run->eos.gamma = c.gamma;
    run->eos.p_inf = c.p_inf;
    for (int s = 0; s < 6; ++s) run->bc.type[s] = c.bc[s];
    halo_kinds(c, c.reconstruction == FVG_RECON_WENO5 ? 3 : 2, run->bc.halo);
    for (int h = 0; h < 2; ++h)
        if (run->is_part && run->peer[h]) {   // an interface: the neighbour's cells, no boundary rule
            const int side = 2 * split + h;
            run->bc.halo[side] = kHaloPeer;
            run->bc.type[side] = kBcPeriodic;
            run->bc.ext[side] = depth;
        }
    run->bc.u_in = c.u_in;
    run->bc.v_in = c.v_in;
    run->bc.p_out = c.p_out;
    set_body_force(c, run->bc);
    set_nrbc(*cfg, run->bc);   // the whole mesh's lengths and cell sizes
    const int TX = run->dim == 3 ? Tile<3>::X : Tile<2>::X, TY = run->dim == 3 ? Tile<3>::Y : Tile<2>::Y, TZ = run->dim == 3 ? Tile<3>::Z : 1;
    run->tiles[0] = (c.nx + TX - 1) / TX;
    run->tiles[1] = (c.ny + TY - 1) / TY;
    run->tiles[2] = (c.nz + TZ - 1) / TZ;
    run->nb = run->tiles[0] * run->tiles[1] * run->tiles[2];
    const int vt = run->dim == 3 ? 8 : kVisc2T;   // viscous tiles: 8^3, or 16 x 16 in 2-D
    run->ntiles_v[0] = (c.nx + vt - 1) / vt;
    run->ntiles_v[1] = (c.ny + vt - 1) / vt;
    run->ntiles_v[2] = run->dim == 3 ? (c.nz + 7) / 8 : 1;
    run->nbv = run->ntiles_v[0] * run->ntiles_v[1] * run->ntiles_v[2];
    const int hx = run->dim == 3 ? 8 : 16, hz = run->dim == 3 ? 4 : 1;   // MUSCL-Hancock tiles
    run->ntiles_h[0] = (c.nx + hx - 1) / hx;
    run->ntiles_h[1] = (c.ny + hx - 1) / hx;
    run->ntiles_h[2] = (c.nz + hz - 1) / hz;
    run->nbh = run->ntiles_h[0] * run->ntiles_h[1] * run->ntiles_h[2];
    bool full = run->is_part || c.positivity_fallback || c.use_bodyforce || run->src_on;
    for (int s = 0; s < 6; ++s) full = full || c.bc[s] == FVG_BC_NONREFLECTING;
    run->full = full;
    run->stage = run->dim == 3 ? stage_launcher<3>(c.reconstruction, c.riemann, full) : stage_launcher<2>(c.reconstruction, c.riemann, full);
    if (c.precision == FVG_PREC_MIXED) {
        const MixedStage ms = mixed_stage(run->dim, c.reconstruction, c.riemann, full);
        run->stage.prepare = ms.prepare;
        run->stage.launch = ms.launch;
        if (c.use_viscous && mixed_viscous_prepare() != cudaSuccess) {
            run->err = "kernel set-up failed (shared-memory limit)";
            return bail(FVG_ERR_CUDA);
        }
    }
    // the seed residual of MUSCL-Hancock and every residual use the stage kernel; the viscous and predictor kernels as needed
    if (run->stage.prepare() != cudaSuccess || (c.use_viscous && (run->dim == 3 ? prepare_viscous() : prepare_viscous2d()) != cudaSuccess) ||
        (c.reconstruction == FVG_RECON_MUSCL && prepare_hancock(c.riemann == FVG_RIEMANN_LOWMACH ? kLowMach : kHLLC, full, run->dim) != cudaSuccess)) {
        run->err = "kernel set-up failed (shared-memory limit)";
        return bail(FVG_ERR_CUDA);
    }
    const size_t sbytes = sizeof(double) * run->m.plane * run->nvar;
    if (cudaStreamCreateWithFlags(&run->stream, cudaStreamNonBlocking) != cudaSuccess || cudaMalloc(&run->U, sbytes) != cudaSuccess ||
        cudaMalloc(&run->Ut, sbytes) != cudaSuccess || cudaMalloc(&run->R, sbytes) != cudaSuccess ||
        (c.use_viscous && cudaMalloc(&run->Rv, sbytes) != cudaSuccess) || cudaMalloc(&run->ctl, sizeof(Ctl)) != cudaSuccess ||
        cudaMalloc(&run->bm_seed, sizeof(double) * run->nb) != cudaSuccess ||
        (run->is_part && (cudaMalloc(&run->xbuf, sizeof(double) * 4 * run->xcount) != cudaSuccess || cudaMalloc(&run->xred, sizeof(double) * 2) != cudaSuccess))) {
        run->err = "device allocation failed";
        return bail(FVG_ERR_CUDA);
    }
    // the state arrays start with the ghost planes: U, Ut, R, Rv point at the first interior plane
    for (double** p : {&run->U, &run->Ut, &run->R, &run->Rv})
        if (*p) cudaMemsetAsync(*p, 0, sbytes, run->stream), *p += run->goff;
    if (run->xred) cudaMemsetAsync(run->xred, 0, sizeof(double) * 2, run->stream);
    build_tma_maps(run);
    if (c.positivity_fallback) {
        if (cudaMalloc(&run->fb_flags, run->m.ncells) != cudaSuccess || cudaMalloc(&run->fb_grew, sizeof(int)) != cudaSuccess) {
            run->err = "device allocation failed";
            return bail(FVG_ERR_CUDA);
        }
        cudaMemsetAsync(run->fb_flags, 0, run->m.ncells, run->stream);
    }
    for (int s = 0; s < 2 * (run->dim == 3 ? 3 : 2); ++s)
        if (c.bc[s] == FVG_BC_MASSFLOWINLET && !run->d_utarget) {
            if (cudaMalloc(&run->d_utarget, sizeof(double) * 6) != cudaSuccess) {
                run->err = "device allocation failed";
                return bail(FVG_ERR_CUDA);
            }
            cudaMemsetAsync(run->d_utarget, 0, sizeof(double) * 6, run->stream);
            run->bc.u_target = run->d_utarget;
        }
    if (const int rc = upload_expressions(run, prog)) return bail(rc);
    if (c.flux_quadrature == 1) {   // the face arrays: per axis 6 x nvar doubles and 3 flag bytes per face
        run->fourth = true;
        FourthArgs& fa = run->fa;
        fa.shock_blend = c.shock_blend;
        fa.weno_eps = c.weno_epsilon;
        size_t bytes = 0;
        for (int a = 0; a < run->dim; ++a) {
            fa.periodic[a] = c.bc[2 * a] == FVG_BC_PERIODIC && c.bc[2 * a + 1] == FVG_BC_PERIODIC;
            fa.nf[a] = (long long)(c.nx + (a == 0)) * (c.ny + (a == 1)) * (c.nz + (a == 2));
            bytes += (size_t)fa.nf[a] * (6 * run->nvar * sizeof(double) + 3);
        }
        bytes += 256 * 9 * 3;
        if (cudaMalloc(&run->d_fourth, bytes) != cudaSuccess) {
            run->err = "device allocation of the fourth-order face arrays failed";
            return bail(FVG_ERR_CUDA);
        }
        char* p = static_cast<char*>(run->d_fourth);
        auto take = [&](size_t n) {
            char* q = p;
            p += (n + 255) / 256 * 256;
            return q;
        };
        for (int a = 0; a < run->dim; ++a) {
            const size_t nd = (size_t)fa.nf[a] * run->nvar * sizeof(double);
            fa.UL[a] = reinterpret_cast<double*>(take(nd));
            fa.UR[a] = reinterpret_cast<double*>(take(nd));
            fa.AL[a] = reinterpret_cast<double*>(take(nd));
            fa.AR[a] = reinterpret_cast<double*>(take(nd));
            fa.Fp[a] = reinterpret_cast<double*>(take(nd));
            fa.F[a] = reinterpret_cast<double*>(take(nd));
            fa.good[a] = reinterpret_cast<unsigned char*>(take(fa.nf[a]));
            fa.pt[a] = reinterpret_cast<unsigned char*>(take(fa.nf[a]));
            fa.full[a] = reinterpret_cast<unsigned char*>(take(fa.nf[a]));
        }
    }
    const int nbmax = run->nb > run->nbh ? run->nb : run->nbh;
    for (int s = 0; s < 3; ++s)
        if (cudaMalloc(&run->bm[s], sizeof(double) * nbmax) != cudaSuccess || cudaMalloc(&run->bmv[s], sizeof(double) * run->nbv) != cudaSuccess) {
            run->err = "device allocation failed";
            return bail(FVG_ERR_CUDA);
        }
    if (c.use_ibm) {
        const std::string msg = build_ibm(c, run->tab);
        if (!msg.empty()) {
            run->err = msg;
            return bail(FVG_ERR_CONFIG);
        }
        run->ibm = true;
        if (c.ibm_shape == 2) {   // (enable_motion: the reach of the section about the pivot)
            std::string err;
            run->ref_poly = place_section(c, err);
            for (size_t q = 0; q < run->ref_poly.size() / 2; ++q)
                run->reach = vmax(run->reach, std::hypot(run->ref_poly[2 * q] - c.ibm_cx, run->ref_poly[2 * q + 1] - c.ibm_cy));
            run->cfg.ibm_section = nullptr;   // (the caller's memory is not kept)
        }
        run->dynamic = c.ibm_mass > 0.0 || c.ibm_inertia > 0.0;
        run->moving = run->dynamic || c.ibm_vx != 0.0 || c.ibm_vy != 0.0 || c.ibm_vz != 0.0 || c.ibm_omega != 0.0 || c.ibm_omega_x != 0.0 ||
                      c.ibm_omega_y != 0.0;
        if (run->dynamic) {   // it starts at its placement with the velocities given (Simulation.cpp:301-312)
            if (c.ibm_mass > 0.0) {
                run->body.u = c.ibm_vx;
                run->body.v = c.ibm_vy;
                run->body.w = c.ibm_vz;
            }
            if (c.ibm_inertia > 0.0) {
                run->body.om = c.ibm_omega;
                run->body.omx = c.ibm_omega_x;
                run->body.omy = c.ibm_omega_y;
            }
            if (c.ibm_cm_x != 0.0 || c.ibm_cm_y != 0.0) {   // body frame to mesh axes: a section is placed turned by ibm_aoa, nose up
                const double a = c.ibm_shape == 2 ? c.ibm_aoa * std::acos(-1.0) / 180.0 : 0.0, ca = std::cos(a), sa = std::sin(a);
                run->cm0[0] = c.ibm_cm_x * ca + c.ibm_cm_y * sa;
                run->cm0[1] = -c.ibm_cm_x * sa + c.ibm_cm_y * ca;
            }
            if (cudaMalloc(&run->d_bload, sizeof(double) * 6) != cudaSuccess || cudaMemset(run->d_bload, 0, sizeof(double) * 6) != cudaSuccess) {
                run->err = "device allocation failed";
                return bail(FVG_ERR_CUDA);
            }
        }
        if (const int rc = upload_ibm(run)) return bail(rc);
    }
    Ctl h{};
    h.cfl = c.cfl;
    h.L = run->L;
    h.dt_max = c.dt_max;
    h.always = 1;
    h.t_end = 0.0;
    cudaMemcpyAsync(run->ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, run->stream);
    if (cudaStreamSynchronize(run->stream) != cudaSuccess) {
        run->err = "device initialisation failed";
        return bail(FVG_ERR_CUDA);
    }
    *out = run;
    return FVG_OK;
}

// The body_pose entries of the reference's checkpoint (Simulation::body_checkpoint, cpp/src/SimulationRestart.cpp:87-97):
// the pose the geometry was built at (x, y, angle), the state of a body driven by the flow (x, y, u, v, ax, ay, dt: zeros
// for a body in prescribed motion), on a 3-D mesh then (z of the geometry, z, w, az), with a driven rotation then (angle,
// angular velocity, its last acceleration) and on a 3-D mesh the x and y components (omega_x, omega_y, their accelerations).
std::vector<double> body_checkpoint(const fvg_run* r) {
    if (!r->moving) return {};
    const fvg_run::Pose& g = r->built;
    const fvg_run::Body& b = r->body;
    const bool d3 = r->dim == 3;
    std::vector<double> v = {g.x, g.y, g.angle, b.x, b.y, b.u, b.v, b.ax, b.ay, b.dt};
    if (d3) v.insert(v.end(), {g.z, b.z, b.w, b.az});
    if (r->cfg.ibm_inertia > 0.0) {
        v.insert(v.end(), {b.th, b.om, b.aom});
        if (d3) v.insert(v.end(), {b.omx, b.omy, b.aomx, b.aomy});
    }
    return v;
}

}   // namespace

extern "C" {

int fvg_destroy(fvg_run* run) {
    if (!run) return FVG_OK;
    cudaSetDevice(run->cfg.device);
    if (run->stream) cudaStreamSynchronize(run->stream);
    for (cudaEvent_t e : run->t_stage.ev) cudaEventDestroy(e);
    for (cudaEvent_t e : run->t_visc.ev) cudaEventDestroy(e);
    for (int g = 0; g < 2; ++g)
        if (run->graph[g]) cudaGraphExecDestroy(run->graph[g]);
    for (double* p : {run->U, run->Ut, run->R, run->Rv})   // the arrays start goff doubles before the first interior plane
        if (p) cudaFree(p - run->goff);
    for (double* p : {run->staging, run->bm_seed, run->bm[0], run->bm[1], run->bm[2], run->bmv[0], run->bmv[1], run->bmv[2], run->xbuf, run->xred,
                      run->d_utarget, run->d_pool, run->d_src, run->d_tv})
        if (p) cudaFree(p);
    if (run->ctl) cudaFree(run->ctl);
    if (run->d_code) cudaFree(run->d_code);
    if (run->d_fourth) cudaFree(run->d_fourth);
    if (run->fb_flags) cudaFree(run->fb_flags);
    if (run->fb_grew) cudaFree(run->fb_grew);
    if (run->sens) cudaFree(run->sens);
    if (run->sens_count) cudaFree(run->sens_count);
    if (run->sens_flags) cudaFree(run->sens_flags);
    if (run->sens_tiles) cudaFree(run->sens_tiles);
    for (void* p : {(void*)run->d_mask, (void*)run->d_slot, (void*)run->d_forced, (void*)run->d_ghost, (void*)run->d_img_cell, (void*)run->d_img_w,
                    (void*)run->d_ratio, (void*)run->d_gn, (void*)run->d_deep, (void*)run->d_solid, (void*)run->d_loads, (void*)run->d_gvel,
                    (void*)run->d_dvel, (void*)run->d_bload, (void*)run->d_span, (void*)run->d_mon})
        if (p) cudaFree(p);
    for (cudaEvent_t e : run->ev_host) cudaEventDestroy(e);
    if (run->xfer) cudaStreamDestroy(run->xfer);
    if (run->stream) cudaStreamDestroy(run->stream);
    delete run;
    return FVG_OK;
}

static int ensure_staging(fvg_run* run) {
    if (run->staging) return FVG_OK;
    CK(cudaMalloc(&run->staging, sizeof(double) * 5 * run->m.ncells));
    return FVG_OK;
}

int fvg_upload_state(fvg_run* run, const double* U, size_t ncells) {
    if (!run || !U) return FVG_ERR_ARGUMENT;
    if ((long long)ncells != run->m.ncells) return fail(run, FVG_ERR_ARGUMENT, "ncells is not the mesh's");
    CK(cudaSetDevice(run->cfg.device));
    int rc = ensure_staging(run);
    if (rc) return rc;
    CK(cudaMemcpyAsync(run->staging, U, sizeof(double) * 5 * ncells, cudaMemcpyHostToDevice, run->stream));
    int* bad = reinterpret_cast<int*>(run->bm_seed);
    CK(cudaMemsetAsync(bad, 0, sizeof(int), run->stream));
    run->cur = 0;
    k_aos_to_planes<<<axpy_blocks(run), 256, 0, run->stream>>>(run->staging, run->U, run->m.plane, run->m.ncells, run->nvar, bad);
    CK(cudaGetLastError());
    int hbad = 0;
    CK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, run->stream));
    CK(cudaStreamSynchronize(run->stream));
    if (hbad) return fail(run, FVG_ERR_STATE, "rho w must be zero on a 2-D mesh");
    return FVG_OK;
}

int fvg_download_state(fvg_run* run, double* U, size_t ncells) {
    if (!run || !U) return FVG_ERR_ARGUMENT;
    if ((long long)ncells != run->m.ncells) return fail(run, FVG_ERR_ARGUMENT, "ncells is not the mesh's");
    CK(cudaSetDevice(run->cfg.device));
    int rc = ensure_staging(run);
    if (rc) return rc;
    k_planes_to_aos<<<axpy_blocks(run), 256, 0, run->stream>>>(run->Ucur(), run->staging, run->m.plane, run->m.ncells, run->nvar);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(U, run->staging, sizeof(double) * 5 * ncells, cudaMemcpyDeviceToHost, run->stream));
    CK(cudaStreamSynchronize(run->stream));
    return FVG_OK;
}

int fvg_residual(fvg_run* run, double predictor_half_dt, double* R, size_t ncells, double* smax) {
    if (!run) return FVG_ERR_ARGUMENT;
    if (run->is_part) return fail(run, FVG_ERR_CONFIG, "a part of a decomposed mesh steps through fvg_part_phase");
    if (R && (long long)ncells != run->m.ncells) return fail(run, FVG_ERR_ARGUMENT, "ncells is not the mesh's");
    CK(cudaSetDevice(run->cfg.device));
    Ctl* c = run->ctl;
    const int* always = &c->always;
    double* out = run->cur ? run->U : run->Ut;   // a buffer that is not the state
    CK(cudaMemsetAsync(&c->status, 0, sizeof(int), run->stream));
    // the stage time: fvg_set_stage_time's, else t (plus half the step for the MUSCL-Hancock predictor)
    const int kind = !std::isnan(run->res_time) ? 3 : (predictor_half_dt > 0.0 ? 4 : 0);
    if (predictor_half_dt > 0.0) {
        if (run->cfg.reconstruction != FVG_RECON_MUSCL)
            return fail(run, FVG_ERR_CONFIG, "the MUSCL-Hancock predictor needs a MUSCL run");
        CK(cudaMemcpyAsync(&c->half_dt, &predictor_half_dt, sizeof(double), cudaMemcpyHostToDevice, run->stream));
        CK(stage_values(run, kind, always));
        if (run->ibm) CK(ibm_fill(run, run->Ucur(), nullptr, 0, always));
        CK(massflow_targets(run, run->Ucur(), always));
        if (run->cfg.use_viscous) CK(launch_visc(run, run->Ucur(), run->bmv[0], always));
        CK(launch_hancock(run, hancock_args(run, run->Ucur(), out, kStoreR, run->bm[0], always)));
        k_stage_max<<<1, 1024, 0, run->stream>>>(c, always, 0, run->bm[0], run->nbh, run->bmv[0], run->cfg.use_viscous ? run->nbv : 0);
    } else {
        CK(refresh_gate(run, run->Ucur(), nullptr));
        run->res_kind = kind;
        const cudaError_t e = residual_stage(run, run->Ucur(), nullptr, out, kStoreR, 0, 0, 0, always);
        run->res_kind = -1;
        CK(e);
        k_stage_max<<<1, 1024, 0, run->stream>>>(c, always, 0, run->bm[0], run->nb, run->bmv[0], run->cfg.use_viscous ? run->nbv : 0);
    }
    CK(cudaGetLastError());
    Ctl h;
    int rc = read_ctl(run, &h);
    if (rc) return rc;
    if (h.status == 5) return fail(run, FVG_ERR_CUDA, "a TMA copy of a stage tile did not complete");
    if (h.status == 6) return fail(run, FVG_ERR_CUDA, "a tensor-core step of the sensor did not complete");
    if (h.status == 3) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "time-dependent boundary values: not finite, or rho_in or p_out not positive, at t = %.17g", h.stage_t);
        return fail(run, FVG_ERR_BOUNDARY, msg);
    }
    if (smax) *smax = h.s_stage[0];
    if (R) {
        if ((rc = ensure_staging(run))) return rc;
        k_planes_to_aos<<<axpy_blocks(run), 256, 0, run->stream>>>(out, run->staging, run->m.plane, run->m.ncells, run->nvar);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(R, run->staging, sizeof(double) * 5 * ncells, cudaMemcpyDeviceToHost, run->stream));
        CK(cudaStreamSynchronize(run->stream));
    }
    return FVG_OK;
}

// The control block's verdict after `done` steps: a time-dependent boundary value out of range, or a diverged step.
static int ctl_status(fvg_run* run, const Ctl& h, int done) {
    // a bounded wait of a kernel that gave up (the run's state is not to be trusted after it)
    if (h.status == 5) return fail(run, FVG_ERR_CUDA, "a TMA copy of a stage tile did not complete");
    if (h.status == 6) return fail(run, FVG_ERR_CUDA, "a tensor-core step of the sensor did not complete");
    if (h.status == 3) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "time-dependent boundary values: not finite, or rho_in or p_out not positive, at t = %.17g (step %d)", h.stage_t,
                      done + 1);
        return fail(run, FVG_ERR_BOUNDARY, msg);
    }
    if (h.status) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "the solution diverged at step %d (t = %.6g, dt = %.3g, largest wave speed = %.3g)", done + 1, h.t, h.dt,
                      h.s_step);
        return fail(run, FVG_ERR_DIVERGED, msg);
    }
    return FVG_OK;
}

static int run_steps(fvg_run* run, double t_end, int max_steps, int use_graph, int* steps) {
    CK(cudaSetDevice(run->cfg.device));
    k_begin<<<1, 1, 0, run->stream>>>(run->ctl, t_end, max_steps);
    CK(cudaGetLastError());
    Ctl h;
    int rc;
    const bool hancock = run->cfg.time_scheme == FVG_TS_HANCOCK;
    int done = 0;
    if (run->moving) {
        // a moving body: step by step, the body placed at the start of each step from the device's clock, the distance
        // it travelled checked after it (at most one cell per step, SimulationRun.cpp:449-458)
        while (true) {
            if ((rc = read_ctl(run, &h))) return rc;
            if (!h.active) break;
            if ((rc = place_body(run, h.t))) return rc;
            cudaError_t e = enqueue_step(run);
            if (e != cudaSuccess) return fail(run, FVG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
            Ctl h2;
            if ((rc = read_ctl(run, &h2))) return rc;
            if (h2.steps == h.steps) {   // the step did not run: the state stayed where it was
                if (hancock) run->cur ^= 1;
                h = h2;
                break;
            }
            const fvg_config& c = run->cfg;
            const double wv[3] = {run->dynamic ? run->body.u : c.ibm_vx, run->dynamic ? run->body.v : c.ibm_vy, run->dynamic ? run->body.w : c.ibm_vz};
            double travel = h2.dt * vmax(fabs(wv[0]) / run->m.dx, fabs(wv[1]) / run->m.dy);
            if (run->dim == 3) travel = vmax(travel, h2.dt * fabs(wv[2]) / run->m.dz);
            if (c.ibm_inertia > 0.0) {   // a driven rotation: how far the section's farthest vertex moves (0 for a circle or sphere)
                const double turn = h2.dt * fabs(run->body.om) * run->reach / vmin(run->m.dx, run->m.dy);
                travel = (c.ibm_cm_x != 0.0 || c.ibm_cm_y != 0.0) ? travel + turn : vmax(travel, turn);
            }
            if (travel > 1.0) {
                if (steps) *steps = h2.steps;
                return fail(run, FVG_ERR_DIVERGED, "the moving body travelled more than one cell in a step (lower the CFL number)");
            }
            if (run->dynamic) {   // the loads of the step's first stage move the body on
                double L[6];
                CK(cudaMemcpy(L, run->d_bload, sizeof(L), cudaMemcpyDeviceToHost));
                fvg_run::Body& b = run->body;
                b.fx = L[0];
                b.fy = L[1];
                b.mz = L[2];
                b.fz = L[3];
                b.mx = L[4];
                b.my = L[5];
                advance_body(run, h2.dt);
            }
            h = h2;
        }
        done = h.steps;
    } else if (!use_graph) {
        // one step at a time (fvg_step)
        cudaError_t e = enqueue_step(run);
        if (e != cudaSuccess) return fail(run, FVG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
        if ((rc = read_ctl(run, &h))) return rc;
        done = h.steps;
        if (hancock && done == 0) run->cur ^= 1;   // the step did not run: the state stayed where it was
    } else if (run->timing) {
        // timed: the same launches, one step at a time, events around the kernels
        const int cur0 = run->cur;
        int chunk = 4, before = 0;
        while (true) {
            const int n = max_steps > 0 ? std::max(1, std::min(chunk, max_steps - before)) : chunk;
            for (int k = 0; k < n; ++k) {
                run->t_stage.step_start.push_back(run->t_stage.used);
                run->t_visc.step_start.push_back(run->t_visc.used);
                cudaError_t e = enqueue_step(run);
                if (e != cudaSuccess) return fail(run, FVG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
            }
            if ((rc = read_ctl(run, &h))) return rc;
            timer_flush(run->t_stage, h.steps - before);
            timer_flush(run->t_visc, h.steps - before);
            before = h.steps;
            if (!h.active) break;
            if (chunk < 64) chunk *= 2;
        }
        done = h.steps;
        // every enqueue flipped the ping-pong; only the steps that ran moved the state
        if (hancock) run->cur = (cur0 + done) & 1;
    } else {
        // a graph of two steps (the MUSCL-Hancock ping-pong returns to its buffer after two), or, with the sensor, of
        // sens_every steps with its refresh in the first (the step count of a run call starts at 0, and a graph
        // advances it by sens_every while the run is active, so the first step of every graph is a refresh step)
        cudaGraphExec_t& graph = run->graph[run->cur];
        if (!graph) {
            const int cur0 = run->cur;
            const int per_graph = run->sens ? run->sens_every : 2;
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(run->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e1 = cudaSuccess;
            for (int k = 0; k < per_graph && e1 == cudaSuccess; ++k) e1 = enqueue_step(run, k == 0);
            cudaError_t e2 = cudaSuccess;
            cudaError_t e3 = cudaStreamEndCapture(run->stream, &g);
            run->cur = cur0;
            if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
                return fail(run, FVG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e1 ? e1 : (e2 ? e2 : e3)));
            CK(cudaGraphInstantiate(&graph, g, 0));
            cudaGraphDestroy(g);
        }
        // graphs in growing chunks between two reads of the clock, never more than a step limit still needs (the steps
        // past it would only be gated off on the device, but their launches cost time)
        const int per_graph = run->sens ? run->sens_every : 2;
        int chunk = 4, ran = 0;
        while (true) {
            const int n = max_steps > 0 ? std::max(1, std::min(chunk, (max_steps - ran + per_graph - 1) / per_graph)) : chunk;
            for (int k = 0; k < n; ++k) CK(cudaGraphLaunch(graph, run->stream));
            if ((rc = read_ctl(run, &h))) return rc;
            if (!h.active) break;
            ran = h.steps;
            if (chunk < 64) chunk *= 2;
        }
        done = h.steps;
        if (hancock && (done & 1)) run->cur ^= 1;
    }
    if (steps) *steps = done;
    return ctl_status(run, h, done);
}

int fvg_step(fvg_run* run, double t_end, double* dt, double* smax) {
    if (!run) return FVG_ERR_ARGUMENT;
    if (run->is_part) return fail(run, FVG_ERR_CONFIG, "a part of a decomposed mesh steps through fvg_part_phase");
    int n = 0;
    const int rc = run_steps(run, t_end, 1, 0, &n);
    if (rc) return rc;
    Ctl h;
    int r2 = read_ctl(run, &h);
    if (r2) return r2;
    if (dt) *dt = n ? h.dt : 0.0;
    if (smax) *smax = n ? h.s_step : 0.0;
    return FVG_OK;
}

int fvg_run_until(fvg_run* run, double t_end, int max_steps, int* steps) {
    if (!run) return FVG_ERR_ARGUMENT;
    if (run->is_part) return fail(run, FVG_ERR_CONFIG, "a part of a decomposed mesh steps through fvg_part_phase");
    return run_steps(run, t_end, max_steps, 1, steps);
}

// ---- one step of a state held in host memory (fvg_step_host)
//
// The state crosses the host link in slabs of planes along the slowest axis (z in 3-D, y in 2-D) on a copy stream. The
// first stage runs tile plane by tile plane as soon as the slabs its cells and their halo read have arrived; the last stage
// runs slab by slab and each finished slab is read back while the next is computed. The launches are those of fvg_step
// (same kernels, same arguments, each over a range of tiles), so the result is bit-identical to upload + fvg_step +
// download.

namespace {

constexpr int kHostSlabs = 16;   // slabs of the state per step at most (events: one per slab and direction)
constexpr int kHostHalo = 3;     // the deepest read beyond a tile along the split axis (WENO5-Z); the viscous sweep reads 1-2

struct HostSlabs {
    int ax = 2, N = 1;     // the split axis and its cells
    long long pc = 1;      // cells of one plane across it (the slab of planes [a, b) is cells [a pc, b pc))
    int planes = 1, n = 1; // planes per slab, slabs
    bool periodic = false;
    int ord[kHostSlabs] = {}, pos[kHostSlabs] = {};   // upload order, and each slab's place in it
};

HostSlabs host_slabs(const fvg_run* r) {
    HostSlabs s;
    s.ax = r->dim == 3 ? 2 : 1;
    s.N = s.ax == 2 ? r->m.nz : r->m.ny;
    s.pc = s.ax == 2 ? (long long)r->m.nx * r->m.ny : r->m.nx;
    const int align = r->dim == 3 ? Tile<3>::Z : 1;
    s.planes = (s.N + kHostSlabs - 1) / kHostSlabs;
    s.planes = std::max(8, (s.planes + align - 1) / align * align);
    s.n = (s.N + s.planes - 1) / s.planes;
    s.periodic = r->cfg.bc[2 * s.ax] == FVG_BC_PERIODIC && r->cfg.bc[2 * s.ax + 1] == FVG_BC_PERIODIC;
    // a periodic axis: the last slab first, so that the first tile plane (which wraps onto it) can start early
    for (int p = 0; p < s.n; ++p) s.ord[p] = s.periodic && s.n > 1 ? (p + s.n - 1) % s.n : p;
    for (int p = 0; p < s.n; ++p) s.pos[s.ord[p]] = p;
    return s;
}

// The upload place after which tile plane j of a kernel with tiles T planes high has every cell it reads: planes
// [jT - H, (j + 1) T + H), wrapped on a periodic axis, else clamped to the mesh (ghost slabs mirror cells inside it).
int slab_need(const HostSlabs& s, int T, int j) {
    int p = 0;
    for (int y = j * T - kHostHalo; y < std::min((j + 1) * T, s.N) + kHostHalo; ++y) {
        const int yy = s.periodic ? ((y % s.N) + s.N) % s.N : std::min(std::max(y, 0), s.N - 1);
        p = std::max(p, s.pos[yy / s.planes]);
    }
    return p;
}

// Runs whose residual reads only cells near each tile: no immersed body (its image points), mass-flow inlet (a whole-side
// sum), positivity fallback (repeats), fourth-order quadrature (face passes); Runge-Kutta and Euler steps.
bool host_pipelined(const fvg_run* r) {
    const int ts = r->cfg.time_scheme;
    return (ts == FVG_TS_EULER || ts == FVG_TS_SSPRK2 || ts == FVG_TS_SSPRK3) && !r->fb_flags && !r->ibm && !r->moving && !r->fourth && !r->is_part &&
           !r->d_utarget;
}

}   // namespace

int fvg_step_host(fvg_run* run, const double* U_in, double* U_out, size_t ncells, double t_end, double* dt, double* smax) {
    if (!run || !U_in || !U_out) return FVG_ERR_ARGUMENT;
    if (run->is_part) return fail(run, FVG_ERR_CONFIG, "a part of a decomposed mesh steps through fvg_part_phase");
    if ((long long)ncells != run->m.ncells) return fail(run, FVG_ERR_ARGUMENT, "ncells is not the mesh's");
    if (!host_pipelined(run)) {   // the same three calls without the overlap
        int rc = fvg_upload_state(run, U_in, ncells);
        if (!rc) rc = fvg_step(run, t_end, dt, smax);
        if (!rc) rc = fvg_download_state(run, U_out, ncells);
        return rc;
    }
    CK(cudaSetDevice(run->cfg.device));
    int rc = ensure_staging(run);
    if (rc) return rc;
    if (!run->xfer) CK(cudaStreamCreateWithFlags(&run->xfer, cudaStreamNonBlocking));
    if (run->ev_host.empty()) {
        run->ev_host.resize(2 * kHostSlabs + 1);
        for (cudaEvent_t& e : run->ev_host) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaEvent_t *ev_up = run->ev_host.data(), *ev_down = ev_up + kHostSlabs, ev_start = ev_up[2 * kHostSlabs];
    const HostSlabs s = host_slabs(run);
    cudaStream_t cs = run->stream, xs = run->xfer;
    Ctl* c = run->ctl;
    const int* act = &c->active;
    const long long pl = run->m.plane;
    const int nv = run->nvar, dim = run->dim, ts = run->cfg.time_scheme;
    const bool visc = run->cfg.use_viscous;
    const int nbv = visc ? run->nbv : 0;
    // the two kernels of a residual, by tile plane along the split axis
    const int Ts = dim == 3 ? Tile<3>::Z : Tile<2>::Y, Tv = dim == 3 ? 8 : kVisc2T;
    const int ns = run->tiles[s.ax], nsv = run->ntiles_v[s.ax];
    const int Ps = run->nb / ns, Pv = run->nbv / nsv;
    auto visc_planes = [&](const double* Uv, double* bmv, int j0, int j1) -> cudaError_t {
        if (!visc || j1 <= j0) return cudaSuccess;
        ViscArgs a = visc_args(run, Uv, bmv, act);
        a.b0 = j0 * Pv;
        const int nblk = (j1 - j0) * Pv;
        return dim == 2 ? launch_viscous2d(a, nblk, cs) : run->cfg.precision == FVG_PREC_MIXED ? mixed_viscous_launch(a, nblk, cs) : launch_viscous(a, nblk, cs);
    };
    auto stage_planes = [&](StageArgs sa, int j0, int j1) -> cudaError_t {
        if (j1 <= j0) return cudaSuccess;
        sa.b0 = j0 * Ps;
        return run->stage.launch(sa, (j1 - j0) * Ps, cs);
    };
    auto slab_cells = [&](int k, long long* c0, long long* cn) {
        *c0 = (long long)k * s.planes * s.pc;
        *cn = (long long)(std::min((k + 1) * s.planes, s.N) - k * s.planes) * s.pc;
    };
    auto flat_blocks = [](long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); };
#define CKL(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(run, FVG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

    // ---- the upload overlapped with the first stage
    int* bad = reinterpret_cast<int*>(run->bm_seed);   // a 2-D mesh given rho w != 0
    CK(cudaMemsetAsync(bad, 0, sizeof(int), cs));
    k_begin<<<1, 1, 0, cs>>>(c, t_end, 1);
    CKL(cudaGetLastError());
    CK(cudaEventRecord(ev_start, cs));   // the staging buffer is free once the run's earlier work is done
    CK(cudaStreamWaitEvent(xs, ev_start, 0));
    run->cur = 0;
    // the sensor refreshes its gate every sens_every steps of these calls, from the whole state
    const bool refresh = run->sens && run->host_steps % run->sens_every == 0;
    std::vector<int> need_v(nsv), need_s(ns);
    for (int j = 0; j < nsv; ++j) need_v[j] = refresh ? s.n - 1 : slab_need(s, Tv, j);
    for (int j = 0; j < ns; ++j) {
        int p = refresh ? s.n - 1 : slab_need(s, Ts, j);
        if (visc)   // and the viscous tile planes of its cells
            for (int v = j * Ts / Tv; v <= (std::min((j + 1) * Ts, s.N) - 1) / Tv; ++v) p = std::max(p, need_v[v]);
        need_s[j] = p;
    }
    CKL(stage_values(run, run->res_kind >= 0 ? run->res_kind : 0, act));
    const StageArgs sa1 = stage_args(run, run->U, nullptr, run->R, kStoreR, 0, 0, visc ? run->Rv : nullptr, run->bm[0], act);
    for (int p = 0; p < s.n; ++p) {
        long long c0, cn;
        slab_cells(s.ord[p], &c0, &cn);
        CK(cudaMemcpyAsync(run->staging + 5 * c0, U_in + 5 * c0, sizeof(double) * 5 * cn, cudaMemcpyHostToDevice, xs));
        CK(cudaEventRecord(ev_up[p], xs));
        CK(cudaStreamWaitEvent(cs, ev_up[p], 0));
        k_aos_to_planes<<<flat_blocks(cn), 256, 0, cs>>>(run->staging + 5 * c0, run->U + c0, pl, cn, nv, bad);
        CKL(cudaGetLastError());
        if (refresh && p == s.n - 1) CKL(refresh_gate(run, run->U, nullptr));
        // the tile planes whose reads are complete now, in runs of consecutive planes
        for (int pass = 0; pass < 2; ++pass) {
            const std::vector<int>& need = pass ? need_s : need_v;
            for (int j = 0; j < (int)need.size();) {
                if (need[j] != p) {
                    ++j;
                    continue;
                }
                int k = j;
                while (k < (int)need.size() && need[k] == p) ++k;
                CKL(pass ? stage_planes(sa1, j, k) : visc_planes(run->U, run->bmv[0], j, k));
                j = k;
            }
        }
    }
    k_stage1_dt<<<1, 1024, 0, cs>>>(c, run->bm[0], run->nb, run->bmv[0], nbv);
    CKL(cudaGetLastError());

    // ---- the middle stages, then the last stage overlapped with the download
    auto download = [&](int k) -> int {
        long long c0, cn;
        slab_cells(k, &c0, &cn);
        k_planes_to_aos<<<flat_blocks(cn), 256, 0, cs>>>(run->U + c0, run->staging + 5 * c0, pl, cn, nv);
        CKL(cudaGetLastError());
        CK(cudaEventRecord(ev_down[k], cs));
        CK(cudaStreamWaitEvent(xs, ev_down[k], 0));
        CK(cudaMemcpyAsync(U_out + 5 * c0, run->staging + 5 * c0, sizeof(double) * 5 * cn, cudaMemcpyDeviceToHost, xs));
        return FVG_OK;
    };
    if (ts == FVG_TS_EULER) {
        k_axpy<<<axpy_blocks(run), 256, 0, cs>>>(c, run->U, run->U, run->R, pl, run->m.ncells, nv);
        k_end_rk<<<1, 1, 0, cs>>>(c, 1);
        CKL(cudaGetLastError());
        for (int k = 0; k < s.n; ++k)
            if ((rc = download(k))) return rc;
    } else {
        k_axpy<<<axpy_blocks(run), 256, 0, cs>>>(c, run->Ut, run->U, run->R, pl, run->m.ncells, nv);
        CKL(cudaGetLastError());
        const double* Ulast = run->Ut;
        double ca = 0.5, cb = 0.5;
        int st = 1;
        if (ts == FVG_TS_SSPRK3 && !run->tv_on && !run->src_unsteady) {
            // stages 2 and 3 as a wavefront over the tile planes, each slab downloaded as soon as its cells are final, so
            // the download overlaps both stages. Stage 3 on a tile plane reads stage 2's state R up to kHostHalo cells
            // beyond it (wrapped on a periodic axis) and its viscous sweep R one cell beyond its viscous tiles; a viscous
            // sweep of stage 3 overwrites the viscous residual Rv of its tiles only once every stage-2 tile plane over
            // them has read it. (Without per-stage boundary values or sources: one array holds those for the stage.)
            const StageArgs sa2 = stage_args(run, run->Ut, run->U, run->R, kCombine, 0.75, 0.25, visc ? run->Rv : nullptr, run->bm[1], act);
            const StageArgs sa3 = stage_args(run, run->R, run->U, run->U, kCombine, 1.0 / 3.0, 2.0 / 3.0, visc ? run->Rv : nullptr, run->bm[2], act);
            std::vector<char> done2(ns, 0), done2v(nsv, 0), done3v(nsv, 0);
            auto plane_of = [&](int y, int T) { return (s.periodic ? ((y % s.N) + s.N) % s.N : std::min(std::max(y, 0), s.N - 1)) / T; };
            // stage 2 on every tile plane over cells [lo, hi) not run yet (its viscous tiles first), in runs of consecutive planes
            auto ensure2 = [&](int lo, int hi) -> int {
                std::vector<char> want(ns, 0);
                for (int y = lo; y < hi; ++y) want[plane_of(y, Ts)] = 1;
                for (int j = 0; j < ns;) {
                    if (!want[j] || done2[j]) {
                        ++j;
                        continue;
                    }
                    int k = j;
                    while (k < ns && want[k] && !done2[k]) ++k;
                    const int v0 = j * Ts / Tv, v1 = (std::min(k * Ts, s.N) - 1) / Tv + 1;
                    for (int v = v0; v < v1;) {
                        if (done2v[v]) {
                            ++v;
                            continue;
                        }
                        int w = v;
                        while (w < v1 && !done2v[w]) done2v[w++] = 1;
                        CKL(visc_planes(run->Ut, run->bmv[1], v, w));
                        v = w;
                    }
                    CKL(stage_planes(sa2, j, k));
                    for (int q = j; q < k; ++q) done2[q] = 1;
                    j = k;
                }
                return FVG_OK;
            };
            int j3 = 0, kd = 0;
            for (int k = 0; k < s.n; ++k) {
                // stage 3 on every tile plane with a cell in slabs 0 .. k
                const int j_end = (std::min((k + 1) * s.planes, s.N) + Ts - 1) / Ts;
                if (j_end > j3) {
                    const int c_lo = j3 * Ts, c_hi = std::min(j_end * Ts, s.N);
                    if (visc) {
                        const int v0 = c_lo / Tv, v1 = (c_hi - 1) / Tv + 1;
                        for (int v = v0; v < v1; ++v) {
                            if (done3v[v]) continue;
                            if ((rc = ensure2(v * Tv - 1, std::min((v + 1) * Tv, s.N) + 1))) return rc;
                            CKL(visc_planes(run->R, run->bmv[2], v, v + 1));
                            done3v[v] = 1;
                        }
                    }
                    if ((rc = ensure2(c_lo - kHostHalo, c_hi + kHostHalo))) return rc;
                    CKL(stage_planes(sa3, j3, j_end));
                    j3 = j_end;
                }
                // the slabs whose cells are all final now
                for (; kd < s.n && std::min((kd + 1) * s.planes, s.N) <= std::min(j3 * Ts, s.N); ++kd)
                    if ((rc = download(kd))) return rc;
            }
            for (; kd < s.n; ++kd)
                if ((rc = download(kd))) return rc;
            k_stage_max<<<1, 1024, 0, cs>>>(c, act, 1, run->bm[1], run->nb, run->bmv[1], nbv);
            k_stage_max<<<1, 1024, 0, cs>>>(c, act, 2, run->bm[2], run->nb, run->bmv[2], nbv);
            k_end_rk<<<1, 1, 0, cs>>>(c, 3);
            CKL(cudaGetLastError());
        } else {
        if (ts == FVG_TS_SSPRK3) {
            CKL(stage_values(run, run->res_kind >= 0 ? run->res_kind : 1, act));
            CKL(visc_planes(run->Ut, run->bmv[1], 0, nsv));
            CKL(stage_planes(stage_args(run, run->Ut, run->U, run->R, kCombine, 0.75, 0.25, visc ? run->Rv : nullptr, run->bm[1], act), 0, ns));
            k_stage_max<<<1, 1024, 0, cs>>>(c, act, 1, run->bm[1], run->nb, run->bmv[1], nbv);
            CKL(cudaGetLastError());
            Ulast = run->R;
            ca = 1.0 / 3.0;
            cb = 2.0 / 3.0;
            st = 2;
        }
        CKL(stage_values(run, run->res_kind >= 0 ? run->res_kind : st, act));
        const StageArgs sa = stage_args(run, Ulast, run->U, run->U, kCombine, ca, cb, visc ? run->Rv : nullptr, run->bm[st], act);
        int jv = 0, js = 0;
        for (int k = 0; k < s.n; ++k) {
            // every tile plane with a cell in slabs 0 .. k, and the viscous tile planes of their cells
            const int js_end = (std::min((k + 1) * s.planes, s.N) + Ts - 1) / Ts;
            const int jv_end = (std::min(js_end * Ts, s.N) + Tv - 1) / Tv;
            CKL(visc_planes(Ulast, run->bmv[st], jv, jv_end));
            CKL(stage_planes(sa, js, js_end));
            jv = std::max(jv, jv_end);
            js = std::max(js, js_end);
            if ((rc = download(k))) return rc;
        }
        k_stage_max<<<1, 1024, 0, cs>>>(c, act, st, run->bm[st], run->nb, run->bmv[st], nbv);
        k_end_rk<<<1, 1, 0, cs>>>(c, ts == FVG_TS_SSPRK2 ? 2 : 3);
        CKL(cudaGetLastError());
        }
    }
#undef CKL
    int hbad = 0;
    CK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, cs));
    CK(cudaStreamSynchronize(xs));
    Ctl h;
    if ((rc = read_ctl(run, &h))) return rc;
    if (hbad) return fail(run, FVG_ERR_STATE, "rho w must be zero on a 2-D mesh");
    if (h.steps && run->sens) ++run->host_steps;
    if (dt) *dt = h.steps ? h.dt : 0.0;
    if (smax) *smax = h.steps ? h.s_step : 0.0;
    return ctl_status(run, h, h.steps);
}

int fvg_part_info(const fvg_run* run, int* axis, int* first, int* count, int* depth, int* peer_lo, int* peer_hi) {
    if (!run || !run->is_part) return FVG_ERR_ARGUMENT;
    if (axis) *axis = run->split;
    if (first) *first = run->first;
    if (count) *count = run->count;
    if (depth) *depth = run->depth;
    if (peer_lo) *peer_lo = run->peer[0];
    if (peer_hi) *peer_hi = run->peer[1];
    return FVG_OK;
}

int fvg_part_buffers(fvg_run* run, double** send_lo, double** send_hi, double** recv_lo, double** recv_hi, long long* count, double** reduce) {
    if (!run || !run->is_part) return FVG_ERR_ARGUMENT;
    if (send_lo) *send_lo = run->xbuf;
    if (send_hi) *send_hi = run->xbuf + run->xcount;
    if (recv_lo) *recv_lo = run->xbuf + 2 * run->xcount;
    if (recv_hi) *recv_hi = run->xbuf + 3 * run->xcount;
    if (count) *count = run->xcount;
    if (reduce) *reduce = run->xred;
    return FVG_OK;
}

int fvg_part_begin(fvg_run* run, double t_end, int max_steps) {
    if (!run) return FVG_ERR_ARGUMENT;
    if (!run->is_part) return fail(run, FVG_ERR_CONFIG, "not a part of a decomposed mesh");
    CK(cudaSetDevice(run->cfg.device));
    k_begin<<<1, 1, 0, run->stream>>>(run->ctl, t_end, max_steps);
    CK(cudaGetLastError());
    return FVG_OK;
}

int fvg_part_phase(fvg_run* run, int phase, int* comm, int* nreduce) {
    if (!run || !comm || !nreduce) return FVG_ERR_ARGUMENT;
    if (!run->is_part) return fail(run, FVG_ERR_CONFIG, "not a part of a decomposed mesh");
    CK(cudaSetDevice(run->cfg.device));
    const cudaError_t e = part_phase(run, phase, comm, nreduce);
    if (e != cudaSuccess) return fail(run, FVG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    if (*comm < 0) return fail(run, FVG_ERR_ARGUMENT, "no such phase of this time scheme");
    return FVG_OK;
}

int fvg_part_status(fvg_run* run, int* active, int* steps, double* t, double* dt, double* smax) {
    if (!run) return FVG_ERR_ARGUMENT;
    CK(cudaSetDevice(run->cfg.device));
    Ctl h;
    const int rc = read_ctl(run, &h);
    if (rc) return rc;
    if (active) *active = h.active;
    if (steps) *steps = h.steps;
    if (t) *t = h.t;
    if (dt) *dt = h.dt;
    if (smax) *smax = h.s_step;
    if (h.status == 3) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "time-dependent boundary values: not finite, or rho_in or p_out not positive, at t = %.17g (step %d)", h.stage_t,
                      h.steps + 1);
        return fail(run, FVG_ERR_BOUNDARY, msg);
    }
    if (h.status) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "the solution diverged at step %d (t = %.6g, dt = %.3g, largest wave speed = %.3g)", h.steps + 1, h.t, h.dt, h.s_step);
        return fail(run, FVG_ERR_DIVERGED, msg);
    }
    return FVG_OK;
}

int fvg_get_time(const fvg_run* run, double* t) {
    if (!run || !t) return FVG_ERR_ARGUMENT;
    fvg_run* r = const_cast<fvg_run*>(run);
    Ctl h;
    int rc = read_ctl(r, &h);
    if (rc) return rc;
    *t = h.t;
    return FVG_OK;
}

int fvg_set_time(fvg_run* run, double t) {
    if (!run) return FVG_ERR_ARGUMENT;
    CK(cudaMemcpyAsync(&run->ctl->t, &t, sizeof(double), cudaMemcpyHostToDevice, run->stream));
    CK(cudaStreamSynchronize(run->stream));
    return FVG_OK;
}

int fvg_set_stage_time(fvg_run* run, double t) {
    if (!run) return FVG_ERR_ARGUMENT;
    run->res_time = t;
    return FVG_OK;
}

int fvg_get_lagged_speed(const fvg_run* run, double* s) {
    if (!run || !s) return FVG_ERR_ARGUMENT;
    Ctl h;
    int rc = read_ctl(const_cast<fvg_run*>(run), &h);
    if (rc) return rc;
    *s = h.s_lag;
    return FVG_OK;
}

int fvg_set_lagged_speed(fvg_run* run, double s) {
    if (!run) return FVG_ERR_ARGUMENT;
    CK(cudaMemcpyAsync(&run->ctl->s_lag, &s, sizeof(double), cudaMemcpyHostToDevice, run->stream));
    CK(cudaStreamSynchronize(run->stream));
    return FVG_OK;
}

int fvg_dt_length(const fvg_run* run, double* L) {
    if (!run || !L) return FVG_ERR_ARGUMENT;
    *L = run->L;
    return FVG_OK;
}

int fvg_device_state(fvg_run* run, double** planes, long long* plane, int* nvar) {
    if (!run) return FVG_ERR_ARGUMENT;
    if (planes) *planes = run->Ucur();
    if (plane) *plane = run->m.plane;
    if (nvar) *nvar = run->nvar;
    return FVG_OK;
}

int fvg_stream(fvg_run* run, void** stream) {
    if (!run || !stream) return FVG_ERR_ARGUMENT;
    *stream = run->stream;
    return FVG_OK;
}

int fvg_synchronize(fvg_run* run) {
    if (!run) return FVG_ERR_ARGUMENT;
    CK(cudaStreamSynchronize(run->stream));
    return FVG_OK;
}

int fvg_set_timing(fvg_run* run, int on) {
    if (!run) return FVG_ERR_ARGUMENT;
    run->timing = on != 0;
    run->t_stage.ms = run->t_visc.ms = 0.0;
    run->t_stage.n = run->t_visc.n = 0;
    run->t_stage.used = run->t_visc.used = 0;
    return FVG_OK;
}

int fvg_get_timing(const fvg_run* run, double* stage_ms, long long* stage_launches, double* viscous_ms, long long* viscous_launches) {
    if (!run) return FVG_ERR_ARGUMENT;
    if (stage_ms) *stage_ms = run->t_stage.ms;
    if (stage_launches) *stage_launches = run->t_stage.n;
    if (viscous_ms) *viscous_ms = run->t_visc.ms;
    if (viscous_launches) *viscous_launches = run->t_visc.n;
    return FVG_OK;
}

int fvg_set_sensor(fvg_run* run, const void* weights, float threshold, int every, int radius) {
    if (!run) return FVG_ERR_ARGUMENT;
    CK(cudaSetDevice(run->cfg.device));
    CK(cudaStreamSynchronize(run->stream));
    for (int g = 0; g < 2; ++g)
        if (run->graph[g]) {
            cudaGraphExecDestroy(run->graph[g]);
            run->graph[g] = nullptr;
        }
    if (!weights) {   // back to plain WENO5-Z
        if (!run->sens) return FVG_OK;
        const MixedStage ms = mixed_stage(run->dim, run->cfg.reconstruction, run->cfg.riemann, run->full);
        run->stage.prepare = ms.prepare;
        run->stage.launch = ms.launch;
        cudaFree(run->sens);
        run->sens = nullptr;
        return FVG_OK;
    }
    if (run->cfg.precision != FVG_PREC_MIXED || run->cfg.reconstruction != FVG_RECON_WENO5)
        return fail(run, FVG_ERR_CONFIG, "the sensor gates the mixed-precision WENO5-Z form");
    if (every <= 0) every = 10;   // (10: the refresh costs a third of a stage; measured gains over the ungated step 1.04-1.10x, 0.99-1.07x with 5)
    if (radius < 0) radius = (int)std::ceil(run->cfg.cfl * every) + 1;
    const size_t fbytes = (size_t)run->m.plane * run->dim;
    if (!run->sens) CK(cudaMalloc(&run->sens, sizeof(SensorW)));
    const size_t rbytes = (size_t)run->dim * run->m.nz * run->m.ny * run->tiles[0];   // the gate's row pass (after the flags)
    if (!run->sens_flags) CK(cudaMalloc(&run->sens_flags, fbytes + rbytes));
    if (!run->sens_tiles) CK(cudaMalloc(&run->sens_tiles, (size_t)run->nb * run->dim));
    if (!run->sens_count) {
        CK(cudaMalloc(&run->sens_count, 2 * sizeof(unsigned long long)));
        CK(cudaMemset(run->sens_count, 0, 2 * sizeof(unsigned long long)));
    }
    CK(cudaMemcpy(run->sens, weights, sizeof(SensorW), cudaMemcpyDefault));
    const MixedStage ms = mixed_stage_gated(run->dim, run->cfg.riemann, run->full);
    if (ms.prepare() != cudaSuccess) return fail(run, FVG_ERR_CUDA, "kernel set-up failed (shared-memory limit)");
    run->stage.prepare = ms.prepare;
    run->stage.launch = ms.launch;
    run->sens_theta = threshold;
    run->sens_every = every;
    run->sens_radius = radius;
    run->host_steps = 0;
    return FVG_OK;
}

int fvg_get_sensor_gate(fvg_run* run, unsigned char* cell_flags, unsigned char* tile_flags, int* tile, int* tiles) {
    if (!run) return FVG_ERR_ARGUMENT;
    if (!run->sens) return fail(run, FVG_ERR_CONFIG, "the run has no sensor (fvg_set_sensor)");
    CK(cudaSetDevice(run->cfg.device));
    CK(cudaStreamSynchronize(run->stream));
    const int T[3] = {run->dim == 3 ? Tile<3>::X : Tile<2>::X, run->dim == 3 ? Tile<3>::Y : Tile<2>::Y, run->dim == 3 ? Tile<3>::Z : 1};
    for (int d = 0; d < 3; ++d) {
        if (tile) tile[d] = T[d];
        if (tiles) tiles[d] = run->tiles[d];
    }
    for (int a = 0; a < run->dim && cell_flags; ++a)
        CK(cudaMemcpy(cell_flags + a * run->m.ncells, run->sens_flags + a * run->m.plane, run->m.ncells, cudaMemcpyDeviceToHost));
    if (tile_flags) CK(cudaMemcpy(tile_flags, run->sens_tiles, (size_t)run->nb * run->dim, cudaMemcpyDeviceToHost));
    return FVG_OK;
}

int fvg_get_sensor_counts(fvg_run* run, long long* linear, long long* evaluated, int reset) {
    if (!run) return FVG_ERR_ARGUMENT;
    unsigned long long h[2] = {0, 0};
    if (run->sens_count) {
        CK(cudaSetDevice(run->cfg.device));
        CK(cudaStreamSynchronize(run->stream));
        CK(cudaMemcpy(h, run->sens_count, sizeof(h), cudaMemcpyDeviceToHost));
        if (reset) CK(cudaMemset(run->sens_count, 0, sizeof(h)));
    }
    if (linear) *linear = (long long)h[0];
    if (evaluated) *evaluated = (long long)h[1];
    return FVG_OK;
}

int fvg_ibm_loads(fvg_run* run, double* loads) {
    if (!run || !loads) return FVG_ERR_ARGUMENT;
    if (!run->ibm) return fail(run, FVG_ERR_CONFIG, "the run has no immersed body");
    CK(cudaSetDevice(run->cfg.device));
    // the residual of the current state (after a step the scheme's predictor is off: the plain residual, as the monitor's)
    const int* always = &run->ctl->always;
    double* out = run->cur ? run->U : run->Ut;
    CK(refresh_gate(run, run->Ucur(), nullptr));
    CK(residual_stage(run, run->Ucur(), nullptr, out, kStoreR, 0, 0, 0, always));
    const fvg_config& c = run->cfg;
    const double vol = run->dim == 3 ? run->m.dx * run->m.dy * run->m.dz : run->m.dx * run->m.dy;
    // (the moment centre follows a moving body, SimulationRun.cpp:140-141)
    k_ibm_loads<<<1, 32, 0, run->stream>>>(out, run->Ucur(), run->m.plane, run->d_solid, run->nsolid, vol, run->m.nx, run->m.ny, run->m.dx,
                                           run->m.dy, run->moving ? c.ibm_cx + run->pose.x : c.ibm_cx, run->moving ? c.ibm_cy + run->pose.y : c.ibm_cy,
                                           run->bc.grav[0], run->bc.grav[1], run->bc.grav_on, run->d_loads);
    CK(cudaGetLastError());
    double h[3];
    CK(cudaMemcpyAsync(h, run->d_loads, sizeof(h), cudaMemcpyDeviceToHost, run->stream));
    CK(cudaStreamSynchronize(run->stream));
    // the monitor's coefficients (cpp/src/SimulationRun.cpp:94-103): on q A, A = the diameter (2-D, per unit depth), pi r^2
    // (sphere) or diameter x Lz (3-D cylinder); Cm about (ibm_cx, ibm_cy), nose-up positive
    const double L = c.ibm_shape == 2 ? c.ibm_chord : 2.0 * c.ibm_radius;   // the chord of a section, else the diameter
    const double A = run->dim == 2 ? L : (c.ibm_shape == 1 ? 3.14159265358979323846 * c.ibm_radius * c.ibm_radius : L * c.Lz);
    const double qA = 0.5 * c.rho_in * c.u_in * c.u_in * A;
    loads[0] = h[0];
    loads[1] = h[1];
    loads[2] = h[2];
    loads[3] = qA > 0 ? h[0] / qA : 0.0;
    loads[4] = qA > 0 ? h[1] / qA : 0.0;
    loads[5] = qA > 0 ? -h[2] / (qA * L) : 0.0;
    return FVG_OK;
}

int fvg_get_body_state(const fvg_run* run, double* v, int* n) {
    if (!run || !n) return FVG_ERR_ARGUMENT;
    const std::vector<double> b = body_checkpoint(run);
    if (v) {
        if (*n < (int)b.size()) return fail(const_cast<fvg_run*>(run), FVG_ERR_ARGUMENT, "the body state needs " + std::to_string(b.size()) + " doubles");
        std::copy(b.begin(), b.end(), v);
    }
    *n = (int)b.size();
    return FVG_OK;
}

// Simulation::restore_body_from_checkpoint and ImmersedBoundary::restore_geometry (cpp/src/SimulationRestart.cpp:99-160,
// cpp/src/Physics.cpp:1204-1212): the body's state, and the geometry built at the checkpoint's pose with the wall
// velocities of that moment (a body driven by the flow: its own; a prescribed one: the configured velocities and the
// rotation of the run's time, which set it first). The next step places the body from there.
int fvg_set_body_state(fvg_run* run, const double* v, int n) {
    if (!run || (!v && n)) return FVG_ERR_ARGUMENT;
    if (!run->moving) return fail(run, FVG_ERR_CONFIG, "the run has no moving body (a static body's checkpoint has no pose)");
    const bool d3 = run->dim == 3, rot = run->cfg.ibm_inertia > 0.0;
    const int want = (d3 ? 14 : 10) + (rot ? (d3 ? 7 : 3) : 0);
    if (n != want)
        return fail(run, FVG_ERR_ARGUMENT, "a malformed body pose: " + std::to_string(n) + " entries, this run's has " + std::to_string(want) +
                                                  " (a 2-D pose for a 3-D run, or the reverse, or a driven rotation without its angular state)");
    CK(cudaSetDevice(run->cfg.device));
    Ctl h;
    if (const int rc = read_ctl(run, &h)) return rc;
    fvg_run::Pose g;
    g.x = v[0];
    g.y = v[1];
    g.angle = v[2];
    if (d3) g.z = v[10];
    if (run->dynamic) {
        fvg_run::Body& b = run->body;
        b.x = v[3];
        b.y = v[4];
        b.u = v[5];
        b.v = v[6];
        b.ax = v[7];
        b.ay = v[8];
        b.dt = v[9];
        if (d3) {
            b.z = v[11];
            b.w = v[12];
            b.az = v[13];
        }
        if (rot) {
            const int o = n - (d3 ? 7 : 3);
            b.th = v[o];
            b.om = v[o + 1];
            b.aom = v[o + 2];
            if (d3) {
                b.omx = v[o + 3];
                b.omy = v[o + 4];
                b.aomx = v[o + 5];
                b.aomy = v[o + 6];
            }
        }
        g.u = b.u;
        g.v = b.v;
        g.w = d3 ? b.w : 0.0;
        g.omega = rot ? b.om : 0.0;
        g.omega_x = rot && d3 ? b.omx : 0.0;
        g.omega_y = rot && d3 ? b.omy : 0.0;
    } else {
        const fvg_run::Pose now = prescribed_pose(run->cfg, h.t);
        g.u = run->cfg.ibm_vx;
        g.v = run->cfg.ibm_vy;
        g.w = run->cfg.ibm_vz;
        g.omega = now.omega;
        g.omega_x = now.omega_x;
        g.omega_y = now.omega_y;
    }
    IbmGeom geo;
    IbmTable tb;
    if (const int rc = geometry_at(run, g, geo, tb)) return rc;
    run->tab = std::move(tb);
    run->built = g;
    run->pose = g;
    CK(cudaStreamSynchronize(run->stream));
    if (const int rc = upload_ibm(run)) return rc;
    return upload_velocities(run);
}

// the monitor's volume averages and the enstrophy of the run's current state (fvg_monitor, include/fenice_gpu.h)
constexpr int kMonBlocks = 148 * 4, kMonNT = 256;
int fvg_monitor(fvg_run* run, int order, double* out) {
    if (!run || !out || (order != 0 && order != 1)) return FVG_ERR_ARGUMENT;
    if (run->is_part) return fail(run, FVG_ERR_CONFIG, "fvg_monitor takes a whole mesh: join the parts' states for a decomposed run");
    CK(cudaSetDevice(run->cfg.device));
    if (!run->d_mon) CK(cudaMalloc(&run->d_mon, sizeof(double) * (4 * kMonBlocks + 4)));
    double* res = run->d_mon + 4 * kMonBlocks;
    const double* U = run->Ucur();
    const fvg_config& c = run->cfg;
    int per[3];
    for (int d = 0; d < 3; ++d) per[d] = c.bc[2 * d] == FVG_BC_PERIODIC && c.bc[2 * d + 1] == FVG_BC_PERIODIC;
    if (order == 0) k_monitor_seq<<<1, 1, 0, run->stream>>>(U, run->m.plane, run->m.ncells, run->nvar, res);
    k_monitor_cells<kMonNT><<<kMonBlocks, kMonNT, 0, run->stream>>>(run->m, U, run->nvar, per[0], per[1], per[2], run->d_mon);
    k_monitor_final<<<1, 32, 0, run->stream>>>(run->d_mon, kMonBlocks, run->m.ncells, order == 1, res);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, res, sizeof(double) * 4, cudaMemcpyDeviceToHost, run->stream));
    CK(cudaStreamSynchronize(run->stream));
    return FVG_OK;
}

int fvg_face_flux_batch(fvg_run* run, const double* UL, const double* UR, const int* axis, size_t n, double* F, double* smax) {
    if (!run || !UL || !UR || !axis || !F || !smax) return FVG_ERR_ARGUMENT;
    CK(cudaSetDevice(run->cfg.device));
    double *dUL, *dUR, *dF, *dS;
    int* dA;
    CK(cudaMalloc(&dUL, sizeof(double) * 5 * n));
    CK(cudaMalloc(&dUR, sizeof(double) * 5 * n));
    CK(cudaMalloc(&dF, sizeof(double) * 5 * n));
    CK(cudaMalloc(&dS, sizeof(double) * n));
    CK(cudaMalloc(&dA, sizeof(int) * n));
    CK(cudaMemcpyAsync(dUL, UL, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, run->stream));
    CK(cudaMemcpyAsync(dUR, UR, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, run->stream));
    CK(cudaMemcpyAsync(dA, axis, sizeof(int) * n, cudaMemcpyHostToDevice, run->stream));
    CK(cudaMemsetAsync(dF, 0, sizeof(double) * 5 * n, run->stream));
    const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    // the batch always uses the full 3-D state (rho w kept)
    if (run->cfg.riemann == FVG_RIEMANN_LOWMACH)
        k_face_flux<kLowMach, 5><<<blocks, 256, 0, run->stream>>>(run->eos, run->cfg.shock_blend, dUL, dUR, dA, (long long)n, dF, dS);
    else
        k_face_flux<kHLLC, 5><<<blocks, 256, 0, run->stream>>>(run->eos, run->cfg.shock_blend, dUL, dUR, dA, (long long)n, dF, dS);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(F, dF, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, run->stream));
    CK(cudaMemcpyAsync(smax, dS, sizeof(double) * n, cudaMemcpyDeviceToHost, run->stream));
    CK(cudaStreamSynchronize(run->stream));
    cudaFree(dUL);
    cudaFree(dUR);
    cudaFree(dF);
    cudaFree(dS);
    cudaFree(dA);
    return FVG_OK;
}

}   // extern "C"

// ------------------------------------------------------------------------------------------------ residual without allocation
// fvg_residual_noalloc: the residual of a caller's device state with no device allocation at all, for callers that may
// not call cudaMalloc (an allocator owned by a host framework, a memory pool with a fixed budget, code that runs while
// a caller forbids allocation). Its only scratch, the per-CTA wave-speed maxima and a control block, lives in the
// file-scope array below: a fixed 512 KB + 4 KB that every GPU which loads this library keeps until the process exits.
namespace {

constexpr int kNoAllocMaxCtas = 65536;   // per-CTA maxima the array holds: the largest grid a call may launch
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocScratch {
    Ctl ctl;                               // gate (always = 1), dt = 0, the reduced wave speed
    double pad[(4096 - sizeof(Ctl)) / sizeof(double)];
    double blockmax[kNoAllocMaxCtas];
};
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// the device address of g_noalloc_scratch on each device (null until a call on that device has looked it up); host
// threads making their first call at once may each look it up, and each stores the same address
std::atomic<NoAllocScratch*> g_noalloc_dev[kNoAllocMaxDevices];

__global__ void k_noalloc_begin(NoAllocScratch* s) {
    s->ctl = Ctl{};
    s->ctl.always = 1;
    s->ctl.active = 1;
}

__global__ void k_noalloc_reduce(NoAllocScratch* s, int nb) {
    const double v = block_reduce_max(s->blockmax, nb, s->blockmax, 0);
    if (threadIdx.x == 0) s->ctl.s_stage[0] = v;
}

// the message of a failed call goes where fvg_create_error() reads it (this thread's last failure)
int noalloc_fail(int code, const std::string& msg) {
    g_create_error = msg;
    return code;
}

}   // namespace

extern "C" int fvg_residual_noalloc(const fvg_config* cfg, const double* U, long long plane, double* R, double* smax, void* stream) {
    if (!cfg || !U || !R) return noalloc_fail(FVG_ERR_ARGUMENT, "null argument");
    const std::string v = validate(*cfg);
    if (!v.empty()) return noalloc_fail(FVG_ERR_CONFIG, v);
    if (cfg->precision != FVG_PREC_FP64) return noalloc_fail(FVG_ERR_CONFIG, "fvg_residual_noalloc: the FP64 form only");
    if (cfg->use_ibm) return noalloc_fail(FVG_ERR_CONFIG, "fvg_residual_noalloc: an immersed body needs its tables on the device; use fvg_residual");
    if (cfg->use_viscous) return noalloc_fail(FVG_ERR_CONFIG, "fvg_residual_noalloc: viscous runs need a residual-sized scratch array; use fvg_residual");
    if (cfg->flux_quadrature == 1) return noalloc_fail(FVG_ERR_CONFIG, "fvg_residual_noalloc: flux_quadrature = fourth needs its face arrays; use fvg_residual");
    if (has_expressions(*cfg))
        return noalloc_fail(FVG_ERR_CONFIG, "fvg_residual_noalloc: source terms and time-dependent boundary values need their programs on the device; use fvg_residual");
    for (int s = 0; s < 6; ++s)
        if (cfg->bc[s] == FVG_BC_MASSFLOWINLET)
            return noalloc_fail(FVG_ERR_CONFIG, "fvg_residual_noalloc: a mass-flow inlet needs its target on the device; use fvg_residual");
    const fvg_config& c = *cfg;
    const int dim = c.nz > 1 ? 3 : 2;
    const long long ncells = (long long)c.nx * c.ny * c.nz;
    if (plane < ncells) return noalloc_fail(FVG_ERR_ARGUMENT, "plane is smaller than the cell count");
    const int TX = dim == 3 ? Tile<3>::X : Tile<2>::X, TY = dim == 3 ? Tile<3>::Y : Tile<2>::Y, TZ = dim == 3 ? Tile<3>::Z : 1;
    const long long tiles = (long long)((c.nx + TX - 1) / TX) * ((c.ny + TY - 1) / TY) * ((c.nz + TZ - 1) / TZ);
    if (tiles > kNoAllocMaxCtas) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "fvg_residual_noalloc: the mesh needs %lld tiles, more than the %d its fixed scratch holds "
                                       "(at most %d tiles of %dx%dx%d cells)", tiles, kNoAllocMaxCtas, kNoAllocMaxCtas, TX, TY, TZ);
        return noalloc_fail(FVG_ERR_CONFIG, msg);
    }
    // the call runs on cfg->device, made current on this thread as every entry point does
    const int dev = c.device;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return noalloc_fail(FVG_ERR_CONFIG, "fvg_residual_noalloc: device index out of range");
    if (cudaSetDevice(dev) != cudaSuccess) return noalloc_fail(FVG_ERR_CUDA, "cudaSetDevice failed (no such CUDA device?)");
    bool full = c.positivity_fallback || c.use_bodyforce;   // (the residual of a whole mesh: no part interface)
    for (int s = 0; s < 6; ++s) full = full || c.bc[s] == FVG_BC_NONREFLECTING;
    const StageLauncher launcher = dim == 3 ? stage_launcher<3>(c.reconstruction, c.riemann, full) : stage_launcher<2>(c.reconstruction, c.riemann, full);
    NoAllocScratch* scratch = g_noalloc_dev[dev].load(std::memory_order_acquire);
    if (!scratch) {
        // once per device, with that device current: the device address of the scratch array (the host-side name is not one)
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return noalloc_fail(FVG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        scratch = static_cast<NoAllocScratch*>(p);
        g_noalloc_dev[dev].store(scratch, std::memory_order_release);
    }
    if (launcher.prepare() != cudaSuccess) return noalloc_fail(FVG_ERR_CUDA, "kernel set-up failed (shared-memory limit)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the mesh description (host values only)
    Mesh m{};
    m.nx = c.nx;
    m.ny = c.ny;
    m.nz = c.nz;
    m.ncells = ncells;
    m.plane = plane;
    m.dx = c.Lx / c.nx;
    m.dy = c.Ly / c.ny;
    m.dz = c.Lz / c.nz;
    if (dim == 3) {
        m.area[0] = m.dy * m.dz;
        m.area[1] = m.dx * m.dz;
        m.area[2] = m.dx * m.dy;
        m.inv_cell = 1.0 / (m.dx * m.dy * m.dz);
    } else {
        m.area[0] = m.dy;
        m.area[1] = m.dx;
        m.inv_cell = 1.0 / (m.dx * m.dy);
    }
    StageArgs a{};
    a.m = m;
    for (int q = 0; q < 6; ++q) a.bc.type[q] = c.bc[q];
    halo_kinds(c, c.reconstruction == FVG_RECON_WENO5 ? 3 : 2, a.bc.halo);
    a.bc.u_in = c.u_in;
    a.bc.v_in = c.v_in;
    a.bc.p_out = c.p_out;
    set_body_force(c, a.bc);
    set_nrbc(c, a.bc);
    a.eos.type = c.eos_type;
    a.eos.gamma = c.gamma;
    a.eos.p_inf = c.p_inf;
    a.shock_blend = c.shock_blend;
    a.weno_eps = c.weno_epsilon;
    a.limiter = c.limiter;
    a.mode = kStoreR;
    a.U = U;
    a.out = R;
    a.blockmax = scratch->blockmax;
    a.ctl = &scratch->ctl;
    a.gate = &scratch->ctl.always;
    a.tiles[0] = (c.nx + TX - 1) / TX;
    a.tiles[1] = (c.ny + TY - 1) / TY;
    a.tiles[2] = (c.nz + TZ - 1) / TZ;
    // the control block is written afresh by every call (gate on, dt = 0); each CTA overwrites its own maximum
    k_noalloc_begin<<<1, 1, 0, s>>>(scratch);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = launcher.launch(a, (int)tiles, s);
    if (e == cudaSuccess) {
        k_noalloc_reduce<<<1, 1024, 0, s>>>(scratch, (int)tiles);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && smax) e = cudaMemcpyAsync(smax, &scratch->ctl.s_stage[0], sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return noalloc_fail(FVG_ERR_CUDA, std::string("fvg_residual_noalloc: ") + cudaGetErrorString(e));
    return FVG_OK;
}
