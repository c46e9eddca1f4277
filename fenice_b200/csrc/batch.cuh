// Batched independent problems: hundreds of 2-D meshes of uneven sizes advanced together, each with its own clock and
// step, in one persistent launch per Runge-Kutta stage.
//
// The reference runs one Simulation per case (cpp/src/SimulationRun.cpp:369-444: its serial time loop; batches of
// cases are separate processes). Here the problems of a batch share the scheme (reconstruction, Riemann solver, time
// scheme, precision) and differ in mesh, lengths, boundary conditions, gas and initial state. Their states live in three
// pools (the state U, the stage state Ut, the residual / stage buffer R), problem p's NV planes at offset off_p of each
// pool. A work list of (problem, tile) items covers the tiles of the problems still running; a stage launch has a fixed
// grid (a whole number of CTAs per SM) whose CTAs take the items in turn, so the launch shape and the CUDA graph of a
// step never change while problems finish and drop out of the list. Each problem reduces its stage wave speeds with
// atomicMax on the bits of a non-negative double (their integer order is their value order), so the maxima and every
// dt are the bits the problem gets when it runs alone.
#pragma once

#include "stage.cuh"

namespace fvg {

struct BatchProb {
    Mesh m;
    Bc bc;
    Eos<double> eos;
    double shock_blend, weno_eps;
    int limiter;
    long long off;   // first double of the problem's planes in each pool
};

// per-problem control block (the single run's Ctl for a Runge-Kutta scheme)
struct BatchCtl {
    double t, t_end, dt, dt_max, cfl, L;
    unsigned long long s_bits[3];   // largest wave speed of each stage of the current step (bits of a double >= 0)
    double s_step;                  // largest wave speed of the last step
    int active, steps, max_steps, status;
};

struct BatchWork {
    int prob, tile;
};

struct BatchArgs {
    const BatchProb* prob;
    BatchCtl* ctl;
    const BatchWork* work;
    const int* nwork;
    int mode, stage;
    double ca, cb;
    const double* U;    // pools (see StageArgs: U read with halos, U0 at the cell, out never aliases U)
    const double* U0;
    double* out;
};

// The StageArgs of a work item's problem, built once per item by thread 0 in shared memory.
__device__ __forceinline__ void batch_item_args(const BatchArgs& b, const BatchProb& pr, StageArgs& sa) {
    sa.m = pr.m;
    sa.bc = pr.bc;
    sa.eos = pr.eos;
    sa.shock_blend = pr.shock_blend;
    sa.weno_eps = pr.weno_eps;
    sa.limiter = pr.limiter;
    sa.b0 = 0;
    sa.mode = b.mode;
    sa.ca = b.ca;
    sa.cb = b.cb;
    sa.U = b.U + pr.off;
    sa.U0 = b.U0 ? b.U0 + pr.off : nullptr;
    sa.out = b.out + pr.off;
    sa.Rv = nullptr;
    sa.Rvf = nullptr;
    sa.blockmax = nullptr;
    sa.ctl = nullptr;
    sa.gate = nullptr;
    sa.sens_flags = nullptr;   // (shared memory is not initialised: every pointer a stage sweep may test is set here)
    sa.fb = nullptr;
}

// a problem's stage maximum: the reference's rule `if (s > local) local = s` (a NaN or a zero never enters)
__device__ __forceinline__ void batch_stage_max(BatchCtl* c, int stage, double s) {
    if (s > 0.0) atomicMax(&c->s_bits[stage], (unsigned long long)__double_as_longlong(s));
}

// Tile shapes of the batched stage kernels (the autotuner's choices): cells along x and y, threads per CTA.
struct BatchShape {
    int tx, ty, nt;
};
constexpr int kBatchShapes = 4;
constexpr BatchShape kBatchShape[kBatchShapes] = {{64, 1, 64}, {128, 1, 128}, {256, 1, 256}, {16, 15, 256}};

// Whether the y sweep of a work item takes the thin path: a one-cell-high mesh (a shock tube) whose bottom and top sides
// have no halo. Both y faces of every column are then first-order boundary faces, whose states the general sweep takes
// from the cell and its ghost (side_states + round trip, as BoundaryManager::apply_side does for the reference), never
// from the reconstruction; the thin path computes just those two fluxes per column and skips the stencil load and the
// face reconstruction of the y sweep (3-5 times the work of the x sweep on such a mesh). When both sides copy the cell
// (transmissive, or periodic with one row) the two faces have the same states, so one flux serves both.
__device__ __forceinline__ bool thin_y(const Mesh& m, const Bc& bc) { return m.ny == 1 && bc.halo[2] == kHaloNone && bc.halo[3] == kHaloNone; }
__device__ __forceinline__ bool copy_side(int type) { return type == kBcTransmissive || type == kBcPeriodic; }

template <int RECON, int RIEMANN, int TX, int NT>
__device__ __forceinline__ void thin_y_fp64(const StageArgs& a, double* __restrict__ acc, const int o3[3], double& smax) {
    const Mesh& m = a.m;
    const double A = m.area[1];
    const bool same = copy_side(a.bc.type[2]) && copy_side(a.bc.type[3]);
    for (int c = threadIdx.x; c < TX; c += NT) {
        const int i = o3[0] + c;
        if (i >= m.nx) continue;
        St<double, 4> UL, UR, Fb, Ft;
        side_states<4, false>(m, a.bc, a.eos, a.U, 2, i, 0, 0, UL, UR);
        if constexpr (RECON != kFirstOrder) {
            UL = round_trip(a.eos, UL);
            UR = round_trip(a.eos, UR);
        }
        const double sb = face_flux<RIEMANN>(a.eos, a.shock_blend, UL, UR, 1, Fb);
        double st = sb;
        if (same) {
            Ft = Fb;
        } else {
            side_states<4, false>(m, a.bc, a.eos, a.U, 3, i, 0, 0, UL, UR);
            if constexpr (RECON != kFirstOrder) {
                UL = round_trip(a.eos, UL);
                UR = round_trip(a.eos, UR);
            }
            st = face_flux<RIEMANN>(a.eos, a.shock_blend, UL, UR, 1, Ft);
        }
        if (sb > smax) smax = sb;
        if (st > smax) smax = st;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double d = Ft[q] * A - Fb[q] * A;
            acc[q * TX + c] = acc[q * TX + c] - d;
        }
    }
    __syncthreads();
}

// The FP64 batched stage kernel: stage_kernel's tile sweep and epilogue for each work item the CTA takes.
template <int RECON, int RIEMANN, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) batch_stage_kernel(const BatchArgs b) {
    using S = StageShape<2, RECON, TX, TY, 1>;
    constexpr int NV = S::NV, NC = S::NC;
    extern __shared__ double smem[];
    double* P = smem;
    double* WL = P + S::P_SIZE;
    double* WR = WL + NV * S::NF;
    double* acc = WR + NV * S::NF;
    double* red = acc + NV * NC;
    unsigned char* Sf = reinterpret_cast<unsigned char*>(red + 32);
    __shared__ StageArgs sa;
    const int tid = threadIdx.x;
    const int nw = *b.nwork;
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        const BatchWork it = b.work[w];
        if (tid == 0) batch_item_args(b, b.prob[it.prob], sa);
        __syncthreads();
        const Mesh& m = sa.m;
        const int tx = (m.nx + TX - 1) / TX;
        const int o3[3] = {(it.tile % tx) * TX, (it.tile / tx) * TY, 0};
        double smax = 0.0;
        stage_axis<0, 2, RECON, RIEMANN, TX, TY, 1, NT, false>(sa, P, WL, WR, acc, Sf, o3, smax);
        bool thin = false;
        if constexpr (TY == 1) thin = thin_y(m, sa.bc);
        if (thin)
            thin_y_fp64<RECON, RIEMANN, TX, NT>(sa, acc, o3, smax);
        else
            stage_axis<1, 2, RECON, RIEMANN, TX, TY, 1, NT, false>(sa, P, WL, WR, acc, Sf, o3, smax);
        const double dt = b.ctl[it.prob].dt;
        for (int c = tid; c < NC; c += NT) {
            const int i = o3[0] + c % TX, j = o3[1] + c / TX;
            if (i >= m.nx || j >= m.ny) continue;
            const long long cell = (long long)j * m.nx + i;
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                const double r = acc[q * NC + c] * m.inv_cell;
                const long long e = q * m.plane + cell;
                double o;
                if (sa.mode == kStoreR)
                    o = r;
                else if (sa.mode == kAxpy)
                    o = sa.U[e] + dt * r;
                else
                    o = sa.ca * sa.U0[e] + sa.cb * (sa.U[e] + dt * r);
                sa.out[e] = o;
            }
        }
        const double bm = block_max<NT>(smax, red);
        if (tid == 0) batch_stage_max(&b.ctl[it.prob], b.stage, bm);
        __syncthreads();
    }
}

}   // namespace fvg
