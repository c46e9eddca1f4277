// Host runtime of the batched problems (include/fenice_gpu.h: fvg_batch_*) and the FP64 batched kernels.
//
// A step of every running problem (SSP-RK3; SSP-RK2 and Euler drop stages):
//   stage(U -> R)                              one persistent launch over the work list, each problem's stage-1 maximum
//   dt + axpy                                  per problem dt = cfl L / (s1 + 1e-10) clamped to t_end - t and dt_max
//                                              (TimeScheme.cpp:19-25), Ut = U + dt R on the problem's tiles
//   stage(Ut, U0 = U -> R: 3/4 U0 + 1/4 (Ut + dt R))
//   stage(R,  U0 = U -> U: 1/3 U0 + 2/3 (R + dt R3))
//   end                                        per problem S = max(s1, max(s2, s3)), check_progress, t += dt, whether it
//                                              runs on; then the work list of the problems still running
// Built with the FP64 flags of runtime.cu (IEEE-rounded, no contraction): a problem gets the bits of its single run.
#include "../../include/fenice_gpu.h"
#include "batch.cuh"
#include "batch_api.h"
#include "host_common.h"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

using namespace fvg;

namespace {

constexpr double kDtEps = 1e-10;   // TimeScheme.cpp:19

// ------------------------------------------------------------------------------------------------ control kernels
__global__ void k_batch_begin(BatchCtl* c, int n, double t_end, int max_steps) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        BatchCtl& x = c[p];
        x.t_end = t_end;
        x.max_steps = max_steps;
        x.steps = 0;
        x.status = 0;
        x.s_bits[0] = x.s_bits[1] = x.s_bits[2] = 0ull;
        x.active = (x.t < x.t_end) && (max_steps <= 0 || x.steps < max_steps);
    }
}

__device__ __forceinline__ double sbits(unsigned long long b) { return __longlong_as_double((long long)b); }

// The end of a step (nstages > 0: finish_step of every running problem, as k_end_rk of a single run) and the work list
// of the problems that run the next step, in problem order. One CTA of 1024 threads.
__global__ void __launch_bounds__(1024) k_batch_end(const BatchProb* prob, BatchCtl* ctl, int n, int nstages, int TX, int TY, BatchWork* work,
                                                    int* nwork, int* remaining) {
    __shared__ int sum[1024];
    __shared__ int nact[1024];
    const int tid = threadIdx.x;
    if (nstages > 0)
        for (int p = tid; p < n; p += 1024) {
            BatchCtl& c = ctl[p];
            if (c.active) {
                const double s1 = sbits(c.s_bits[0]), s2 = sbits(c.s_bits[1]), s3 = sbits(c.s_bits[2]);
                const double s = nstages == 1 ? s1 : (nstages == 2 ? vmax(s1, s2) : vmax(s1, vmax(s2, s3)));
                c.s_step = s;
                if (!(isfinite(s) && isfinite(c.dt) && c.t + c.dt > c.t)) {   // check_progress (SimulationInternal.hpp:259-267)
                    c.status = 1;
                    c.active = 0;
                } else {
                    c.t = c.t + c.dt;
                    c.steps += 1;
                    c.active = (c.t < c.t_end) && (c.max_steps <= 0 || c.steps < c.max_steps) && c.status == 0;
                }
            }
            c.s_bits[0] = c.s_bits[1] = c.s_bits[2] = 0ull;
        }
    __syncthreads();
    // thread t lists the problems [t per, (t + 1) per)
    const int per = (n + 1023) / 1024, p0 = tid * per, p1 = min(n, p0 + per);
    int cnt = 0, act = 0;
    for (int p = p0; p < p1; ++p)
        if (ctl[p].active) {
            const Mesh& m = prob[p].m;
            cnt += ((m.nx + TX - 1) / TX) * ((m.ny + TY - 1) / TY);
            ++act;
        }
    sum[tid] = cnt;
    nact[tid] = act;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {   // inclusive scan
        const int a = tid >= o ? sum[tid - o] : 0, b = tid >= o ? nact[tid - o] : 0;
        __syncthreads();
        sum[tid] += a;
        nact[tid] += b;
        __syncthreads();
    }
    int base = sum[tid] - cnt;
    for (int p = p0; p < p1; ++p)
        if (ctl[p].active) {
            const Mesh& m = prob[p].m;
            const int nt = ((m.nx + TX - 1) / TX) * ((m.ny + TY - 1) / TY);
            for (int k = 0; k < nt; ++k) work[base + k] = BatchWork{p, k};
            base += nt;
        }
    if (tid == 1023) {
        *nwork = sum[1023];
        *remaining = nact[1023];
    }
}

// The step dt of each running problem from its stage-1 maximum (k_stage1_dt of a single run; the CTAs of a problem
// compute the same dt and the one of tile 0 stores it), then out = a + dt r on the problem's tiles.
__global__ void k_batch_dt_axpy(const BatchProb* prob, BatchCtl* ctl, const BatchWork* work, const int* nwork, int TX, int TY, double* out,
                                const double* a, const double* r) {
    const int nw = *nwork;
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        const BatchWork it = work[w];
        BatchCtl* c = &ctl[it.prob];
        const double s = sbits(c->s_bits[0]);
        double dt = c->cfl * c->L / (s + kDtEps);
        dt = vmin(dt, c->t_end - c->t);
        if (c->dt_max > 0.0) dt = vmin(dt, c->dt_max);
        if (it.tile == 0 && threadIdx.x == 0) c->dt = dt;
        const Mesh& m = prob[it.prob].m;
        const long long off = prob[it.prob].off;
        const int tx = (m.nx + TX - 1) / TX;
        const int i0 = (it.tile % tx) * TX, j0 = (it.tile / tx) * TY;
        const int nc = TX * TY;
        for (int k = threadIdx.x; k < 4 * nc; k += blockDim.x) {
            const int q = k / nc, cc = k % nc;
            const int i = i0 + cc % TX, j = j0 + cc / TX;
            if (i >= m.nx || j >= m.ny) continue;
            const long long e = off + q * m.plane + (long long)j * m.nx + i;
            out[e] = a[e] + dt * r[e];
        }
    }
}

// the problem a cell of the concatenated state array belongs to (cell_off: n + 1 prefix sums)
__device__ __forceinline__ int batch_find(const long long* cell_off, int n, long long g) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cell_off[mid] <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void k_batch_aos_to_planes(const BatchProb* prob, const long long* cell_off, int n, const double* aos, double* U, int* bad) {
    const long long total = cell_off[n];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
        const int p = batch_find(cell_off, n, g);
        const long long c = g - cell_off[p];
        const BatchProb& pr = prob[p];
        for (int q = 0; q < 4; ++q) U[pr.off + q * pr.m.plane + c] = aos[5 * g + q];
        if (aos[5 * g + 4] != 0.0) atomicOr(bad, 1);
    }
}

__global__ void k_batch_planes_to_aos(const BatchProb* prob, const long long* cell_off, int n, const double* U, double* aos) {
    const long long total = cell_off[n];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
        const int p = batch_find(cell_off, n, g);
        const long long c = g - cell_off[p];
        const BatchProb& pr = prob[p];
        for (int q = 0; q < 4; ++q) aos[5 * g + q] = U[pr.off + q * pr.m.plane + c];
        aos[5 * g + 4] = 0.0;
    }
}

__global__ void k_batch_clear_max(BatchCtl* c, int n) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) c[p].s_bits[0] = c[p].s_bits[1] = c[p].s_bits[2] = 0ull;
}

// ------------------------------------------------------------------------------------------------ FP64 kernel dispatch
template <int SHAPE, int RECON, int RIEMANN> struct FK {
    static constexpr BatchShape sh = kBatchShape[SHAPE];
    using S = StageShape<2, RECON, sh.tx, sh.ty, 1>;
    static constexpr auto kern = batch_stage_kernel<RECON, RIEMANN, sh.tx, sh.ty, sh.nt>;
    static cudaError_t prepare() { return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM_BYTES); }
    static cudaError_t launch(const BatchArgs& a, int grid, cudaStream_t s) {
        kern<<<grid, sh.nt, S::SMEM_BYTES, s>>>(a);
        return cudaGetLastError();
    }
    static int resident() {
        int n = 0;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, sh.nt, S::SMEM_BYTES) == cudaSuccess ? n : 0;
    }
    static BatchStage get() { return {prepare, launch, resident}; }
};
template <int SHAPE, int RECON> BatchStage fpick_r(int riemann) {
    return riemann == kLowMach ? FK<SHAPE, RECON, kLowMach>::get() : FK<SHAPE, RECON, kHLLC>::get();
}
template <int SHAPE> BatchStage fpick_s(int recon, int riemann) {
    switch (recon) {
    case kFirstOrder: return fpick_r<SHAPE, kFirstOrder>(riemann);
    case kMuscl: return fpick_r<SHAPE, kMuscl>(riemann);
    case kWeno3: return fpick_r<SHAPE, kWeno3>(riemann);
    default: return fpick_r<SHAPE, kWeno5>(riemann);
    }
}

}   // namespace

BatchStage fvg::batch_fp64_stage(int shape, int recon, int riemann) {
    switch (shape) {
    case 0: return fpick_s<0>(recon, riemann);
    case 1: return fpick_s<1>(recon, riemann);
    case 2: return fpick_s<2>(recon, riemann);
    default: return fpick_s<3>(recon, riemann);
    }
}

// ------------------------------------------------------------------------------------------------ the batch
struct fvg_batch {
    int n = 0;
    std::vector<fvg_config> cfg;
    std::string err;
    int device = 0, precision = 0, recon = 0, riemann = 0, scheme = 0, nstages = 3;
    cudaStream_t stream = nullptr;
    std::vector<BatchProb> prob;
    std::vector<long long> cell_off;   // n + 1 prefix sums of the problems' cells
    long long pool = 0;                // doubles per pool
    double *U = nullptr, *Ut = nullptr, *R = nullptr, *staging = nullptr;
    BatchProb* d_prob = nullptr;
    BatchCtl* d_ctl = nullptr;
    BatchWork* d_work = nullptr;
    long long* d_cell_off = nullptr;
    int *d_nwork = nullptr, *d_remaining = nullptr, *d_bad = nullptr;
    int* h_remaining = nullptr;   // pinned, 2 slots
    BatchStage kern[kBatchShapes];
    bool kern_ok[kBatchShapes] = {};
    int shape = -1, ctas_per_sm = 0, grid = 0, sms = 148;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 8;
    bool timing = false;
    std::vector<cudaEvent_t> ev;
    size_t ev_used = 0;
    double t_ms = 0.0;
    long long t_n = 0;
    std::vector<BatchCtl> h_ctl;   // after a run
};

namespace {

int bfail(fvg_batch* b, int code, const std::string& msg) {
    b->err = msg;
    return code;
}

#define BK(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return bfail(b, FVG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

thread_local std::string g_batch_create_error;

std::string batch_config_error(const fvg_config* cfgs, int n) {
    if (n < 1) return "a batch needs at least one problem";
    const fvg_config& a = cfgs[0];
    for (int p = 0; p < n; ++p) {
        const fvg_config& c = cfgs[p];
        const std::string e = config_error(c);
        if (!e.empty()) return "problem " + std::to_string(p) + ": " + e;
        if (c.nz != 1) return "problem " + std::to_string(p) + ": batched problems are 2-D (nz = 1)";
        if (c.use_viscous || c.use_ibm || c.use_bodyforce || c.positivity_fallback)
            return "problem " + std::to_string(p) + ": batched problems are inviscid, without an immersed body or a body force";
        for (int s = 0; s < 4; ++s)
            if (c.bc[s] == FVG_BC_MASSFLOWINLET || c.bc[s] == FVG_BC_NONREFLECTING)
                return "problem " + std::to_string(p) + ": batched problems have no mass-flow inlet or non-reflecting outlet";
        if (c.time_scheme == FVG_TS_HANCOCK) return "problem " + std::to_string(p) + ": batched problems use Euler, SSP-RK2 or SSP-RK3";
        if (c.flux_quadrature != 0) return "problem " + std::to_string(p) + ": batched problems use the midpoint flux quadrature";
        if (config_has_expressions(c))
            return "problem " + std::to_string(p) + ": batched problems have no case-file source terms or time-dependent boundary values";
        if (c.reconstruction != a.reconstruction || c.riemann != a.riemann || c.time_scheme != a.time_scheme || c.precision != a.precision ||
            c.device != a.device)
            return "problem " + std::to_string(p) + ": the problems of a batch share reconstruction, Riemann solver, time scheme, precision and device";
    }
    return "";
}

int stages_of(int ts) { return ts == FVG_TS_EULER ? 1 : (ts == FVG_TS_SSPRK2 ? 2 : 3); }

long long items_for(const fvg_batch* b, int shape) {
    long long s = 0;
    const BatchShape sh = kBatchShape[shape];
    for (const BatchProb& p : b->prob) s += (long long)((p.m.nx + sh.tx - 1) / sh.tx) * ((p.m.ny + sh.ty - 1) / sh.ty);
    return s;
}

BatchArgs stage_args(const fvg_batch* b, const double* Uin, const double* U0, double* out, int mode, double ca, double cb, int stage) {
    BatchArgs a{};
    a.prob = b->d_prob;
    a.ctl = b->d_ctl;
    a.work = b->d_work;
    a.nwork = b->d_nwork;
    a.mode = mode;
    a.stage = stage;
    a.ca = ca;
    a.cb = cb;
    a.U = Uin;
    a.U0 = U0;
    a.out = out;
    return a;
}

void ev_mark(fvg_batch* b) {
    if (!b->timing) return;
    if (b->ev_used == b->ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        b->ev.push_back(e);
    }
    cudaEventRecord(b->ev[b->ev_used++], b->stream);
}

void ev_flush(fvg_batch* b) {
    for (size_t k = 0; k + 1 < b->ev_used; k += 2) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, b->ev[k], b->ev[k + 1]) == cudaSuccess) {
            b->t_ms += ms;
            b->t_n += 1;
        }
    }
    b->ev_used = 0;
}

cudaError_t launch_stage(fvg_batch* b, const BatchArgs& a) {
    ev_mark(b);
    const cudaError_t e = b->kern[b->shape].launch(a, b->grid, b->stream);
    ev_mark(b);
    return e;
}

cudaError_t enqueue_end(fvg_batch* b, int nstages) {
    const BatchShape sh = kBatchShape[b->shape];
    k_batch_end<<<1, 1024, 0, b->stream>>>(b->d_prob, b->d_ctl, b->n, nstages, sh.tx, sh.ty, b->d_work, b->d_nwork, b->d_remaining);
    return cudaGetLastError();
}

// the launches of one step of every running problem
cudaError_t enqueue_step(fvg_batch* b) {
    cudaError_t e;
    const BatchShape sh = kBatchShape[b->shape];
    const int ag = b->grid;
    if ((e = launch_stage(b, stage_args(b, b->U, nullptr, b->R, kStoreR, 0, 0, 0)))) return e;
    if (b->scheme == FVG_TS_EULER) {
        k_batch_dt_axpy<<<ag, 256, 0, b->stream>>>(b->d_prob, b->d_ctl, b->d_work, b->d_nwork, sh.tx, sh.ty, b->U, b->U, b->R);
        return enqueue_end(b, 1);
    }
    k_batch_dt_axpy<<<ag, 256, 0, b->stream>>>(b->d_prob, b->d_ctl, b->d_work, b->d_nwork, sh.tx, sh.ty, b->Ut, b->U, b->R);
    if (b->scheme == FVG_TS_SSPRK2) {
        if ((e = launch_stage(b, stage_args(b, b->Ut, b->U, b->U, kCombine, 0.5, 0.5, 1)))) return e;
        return enqueue_end(b, 2);
    }
    if ((e = launch_stage(b, stage_args(b, b->Ut, b->U, b->R, kCombine, 0.75, 0.25, 1)))) return e;
    if ((e = launch_stage(b, stage_args(b, b->R, b->U, b->U, kCombine, 1.0 / 3.0, 2.0 / 3.0, 2)))) return e;
    return enqueue_end(b, 3);
}

void drop_graph(fvg_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

int apply_schedule(fvg_batch* b, int shape, int ctas_per_sm) {
    if (shape < 0 || shape >= kBatchShapes || !b->kern_ok[shape]) return bfail(b, FVG_ERR_ARGUMENT, "no such tile shape");
    const int res = b->kern[shape].resident();
    if (res < 1) return bfail(b, FVG_ERR_CUDA, "the tile shape's kernel does not fit on an SM");
    if (ctas_per_sm <= 0 || ctas_per_sm > res) ctas_per_sm = res;
    drop_graph(b);
    b->shape = shape;
    b->ctas_per_sm = ctas_per_sm;
    b->grid = ctas_per_sm * b->sms;
    return FVG_OK;
}

}   // namespace

extern "C" {

int fvg_batch_destroy(fvg_batch* b) {
    if (!b) return FVG_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    for (void* p : {(void*)b->U, (void*)b->Ut, (void*)b->R, (void*)b->staging, (void*)b->d_prob, (void*)b->d_ctl, (void*)b->d_work,
                    (void*)b->d_cell_off, (void*)b->d_nwork, (void*)b->d_remaining, (void*)b->d_bad})
        if (p) cudaFree(p);
    if (b->h_remaining) cudaFreeHost(b->h_remaining);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return FVG_OK;
}

const char* fvg_batch_last_error(const fvg_batch* b) { return b ? b->err.c_str() : "null batch"; }

int fvg_batch_create(const fvg_config* cfgs, int n, fvg_batch** out) {
    if (!cfgs || !out) {
        *create_error_slot() = "null argument";
        return FVG_ERR_ARGUMENT;
    }
    *out = nullptr;
    const std::string v = batch_config_error(cfgs, n);
    if (!v.empty()) {
        *create_error_slot() = v;
        return FVG_ERR_CONFIG;
    }
    auto* b = new fvg_batch();
    auto bail = [&](int code, const char* msg) {
        *create_error_slot() = b->err.empty() ? msg : b->err;
        fvg_batch_destroy(b);
        return code;
    };
    b->n = n;
    b->cfg.assign(cfgs, cfgs + n);
    const fvg_config& a = cfgs[0];
    b->device = a.device;
    b->precision = a.precision;
    b->recon = a.reconstruction;
    b->riemann = a.riemann;
    b->scheme = a.time_scheme;
    b->nstages = stages_of(a.time_scheme);
    if (cudaSetDevice(b->device) != cudaSuccess) return bail(FVG_ERR_CUDA, "cudaSetDevice failed (no CUDA device?)");
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    b->prob.resize(n);
    b->cell_off.assign(n + 1, 0);
    long long off = 0;
    for (int p = 0; p < n; ++p) {
        const fvg_config& c = cfgs[p];
        BatchProb& pr = b->prob[p];
        pr = BatchProb{};
        Mesh& m = pr.m;
        m.nx = c.nx;
        m.ny = c.ny;
        m.nz = 1;
        m.ncells = (long long)c.nx * c.ny;
        m.plane = (m.ncells + 31) / 32 * 32;
        m.dx = c.Lx / c.nx;   // generate_cartesian_mesh_3d (Core.cpp:20-40), as fvg_create
        m.dy = c.Ly / c.ny;
        m.dz = c.Lz / c.nz;
        m.area[0] = m.dy;
        m.area[1] = m.dx;
        m.area[2] = 0.0;
        m.inv_cell = 1.0 / (m.dx * m.dy);
        for (int s = 0; s < 6; ++s) pr.bc.type[s] = c.bc[s];
        config_halo_kinds(c, c.reconstruction == FVG_RECON_WENO5 ? 3 : 2, pr.bc.halo);
        pr.bc.u_in = c.u_in;
        pr.bc.v_in = c.v_in;
        pr.bc.p_out = c.p_out;
        pr.eos.type = c.eos_type;
        pr.eos.gamma = c.gamma;
        pr.eos.p_inf = c.p_inf;
        pr.shock_blend = c.shock_blend;
        pr.weno_eps = c.weno_epsilon;
        pr.limiter = c.limiter;
        pr.off = off;
        off += 4 * m.plane;
        b->cell_off[p + 1] = b->cell_off[p] + m.ncells;
    }
    b->pool = off;
    long long max_items = 0;
    for (int s = 0; s < kBatchShapes; ++s) {
        b->kern[s] = b->precision == FVG_PREC_MIXED ? batch_mixed_stage(s, b->recon, b->riemann) : batch_fp64_stage(s, b->recon, b->riemann);
        b->kern_ok[s] = b->kern[s].prepare() == cudaSuccess;
        if (b->kern_ok[s]) max_items = std::max(max_items, items_for(b, s));
    }
    cudaGetLastError();
    if (max_items > (1LL << 31) - 1) return bail(FVG_ERR_CONFIG, "too many tiles in the batch");
    std::vector<BatchCtl> hc(n);
    for (int p = 0; p < n; ++p) {
        const fvg_config& c = cfgs[p];
        BatchCtl x{};
        x.cfl = c.cfl;
        x.dt_max = c.dt_max;
        x.L = vmin(c.Lx / c.nx, c.Ly / c.ny);   // 2-D: min(dx, dy) (Simulation.cpp:225-227)
        hc[p] = x;
    }
    const size_t pb = sizeof(double) * (size_t)b->pool;
    bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess && cudaMalloc(&b->U, pb) == cudaSuccess &&
              cudaMalloc(&b->Ut, pb) == cudaSuccess && cudaMalloc(&b->R, pb) == cudaSuccess &&
              cudaMalloc(&b->d_prob, sizeof(BatchProb) * n) == cudaSuccess && cudaMalloc(&b->d_ctl, sizeof(BatchCtl) * n) == cudaSuccess &&
              cudaMalloc(&b->d_work, sizeof(BatchWork) * (size_t)std::max(1LL, max_items)) == cudaSuccess &&
              cudaMalloc(&b->d_cell_off, sizeof(long long) * (n + 1)) == cudaSuccess && cudaMalloc(&b->d_nwork, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&b->d_remaining, sizeof(int)) == cudaSuccess && cudaMalloc(&b->d_bad, sizeof(int)) == cudaSuccess &&
              cudaHostAlloc(&b->h_remaining, 2 * sizeof(int), cudaHostAllocDefault) == cudaSuccess;
    if (!ok) return bail(FVG_ERR_CUDA, "device allocation failed");
    ok = cudaMemcpyAsync(b->d_prob, b->prob.data(), sizeof(BatchProb) * n, cudaMemcpyHostToDevice, b->stream) == cudaSuccess &&
         cudaMemcpyAsync(b->d_ctl, hc.data(), sizeof(BatchCtl) * n, cudaMemcpyHostToDevice, b->stream) == cudaSuccess &&
         cudaMemcpyAsync(b->d_cell_off, b->cell_off.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, b->stream) == cudaSuccess &&
         cudaMemsetAsync(b->U, 0, pb, b->stream) == cudaSuccess && cudaMemsetAsync(b->Ut, 0, pb, b->stream) == cudaSuccess &&
         cudaMemsetAsync(b->R, 0, pb, b->stream) == cudaSuccess && cudaMemsetAsync(b->d_nwork, 0, sizeof(int), b->stream) == cudaSuccess &&
         cudaStreamSynchronize(b->stream) == cudaSuccess;
    if (!ok) return bail(FVG_ERR_CUDA, "device initialisation failed");
    b->h_ctl = hc;
    *out = b;
    return FVG_OK;
}

int fvg_batch_cells(const fvg_batch* b, long long* ncells) {
    if (!b || !ncells) return FVG_ERR_ARGUMENT;
    *ncells = b->cell_off[b->n];
    return FVG_OK;
}

static int ensure_staging(fvg_batch* b) {
    if (b->staging) return FVG_OK;
    BK(cudaMalloc(&b->staging, sizeof(double) * 5 * (size_t)b->cell_off[b->n]));
    return FVG_OK;
}

static int copy_blocks(const fvg_batch* b) {
    const long long n = b->cell_off[b->n];
    const long long g = (n + 255) / 256;
    return (int)std::min<long long>(std::max(1LL, g), 148LL * 16);
}

int fvg_batch_upload(fvg_batch* b, const double* U, size_t ncells) {
    if (!b || !U) return FVG_ERR_ARGUMENT;
    if ((long long)ncells != b->cell_off[b->n]) return bfail(b, FVG_ERR_ARGUMENT, "ncells is not the batch's");
    BK(cudaSetDevice(b->device));
    int rc = ensure_staging(b);
    if (rc) return rc;
    BK(cudaMemcpyAsync(b->staging, U, sizeof(double) * 5 * ncells, cudaMemcpyHostToDevice, b->stream));
    BK(cudaMemsetAsync(b->d_bad, 0, sizeof(int), b->stream));
    k_batch_aos_to_planes<<<copy_blocks(b), 256, 0, b->stream>>>(b->d_prob, b->d_cell_off, b->n, b->staging, b->U, b->d_bad);
    BK(cudaGetLastError());
    int hbad = 0;
    BK(cudaMemcpyAsync(&hbad, b->d_bad, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    if (hbad) return bfail(b, FVG_ERR_STATE, "rho w must be zero on a 2-D mesh");
    return FVG_OK;
}

int fvg_batch_download(fvg_batch* b, double* U, size_t ncells) {
    if (!b || !U) return FVG_ERR_ARGUMENT;
    if ((long long)ncells != b->cell_off[b->n]) return bfail(b, FVG_ERR_ARGUMENT, "ncells is not the batch's");
    BK(cudaSetDevice(b->device));
    int rc = ensure_staging(b);
    if (rc) return rc;
    k_batch_planes_to_aos<<<copy_blocks(b), 256, 0, b->stream>>>(b->d_prob, b->d_cell_off, b->n, b->U, b->staging);
    BK(cudaGetLastError());
    BK(cudaMemcpyAsync(U, b->staging, sizeof(double) * 5 * ncells, cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    return FVG_OK;
}

int fvg_batch_set_schedule(fvg_batch* b, int shape, int ctas_per_sm) {
    if (!b) return FVG_ERR_ARGUMENT;
    BK(cudaSetDevice(b->device));
    return apply_schedule(b, shape, ctas_per_sm);
}

int fvg_batch_get_schedule(const fvg_batch* b, int* shape, int* tile_x, int* tile_y, int* grid) {
    if (!b) return FVG_ERR_ARGUMENT;
    if (shape) *shape = b->shape;
    if (tile_x) *tile_x = b->shape >= 0 ? kBatchShape[b->shape].tx : 0;
    if (tile_y) *tile_y = b->shape >= 0 ? kBatchShape[b->shape].ty : 0;
    if (grid) *grid = b->grid;
    return FVG_OK;
}

int fvg_batch_autotune(fvg_batch* b, int* shape, int* ctas_per_sm, double* stage_ms) {
    if (!b) return FVG_ERR_ARGUMENT;
    BK(cudaSetDevice(b->device));
    const bool timing = b->timing;
    b->timing = false;
    cudaEvent_t e0, e1;
    BK(cudaEventCreate(&e0));
    BK(cudaEventCreate(&e1));
    double best = 1e300;
    int best_s = -1, best_c = 0;
    constexpr int kWarm = 2, kReps = 5;
    for (int s = 0; s < kBatchShapes; ++s) {
        if (!b->kern_ok[s]) continue;
        const int res = b->kern[s].resident();
        for (int cps = 1; cps <= res; ++cps) {
            int rc = apply_schedule(b, s, cps);
            if (rc) continue;
            // every problem's tiles (as if all run), one STORE_R stage into the scratch pool R
            k_batch_begin<<<(b->n + 255) / 256, 256, 0, b->stream>>>(b->d_ctl, b->n, 1e300, 0);
            BK(enqueue_end(b, 0));
            const BatchArgs a = stage_args(b, b->U, nullptr, b->R, kStoreR, 0, 0, 0);
            for (int k = 0; k < kWarm; ++k) BK(b->kern[s].launch(a, b->grid, b->stream));
            BK(cudaEventRecord(e0, b->stream));
            for (int k = 0; k < kReps; ++k) BK(b->kern[s].launch(a, b->grid, b->stream));
            BK(cudaEventRecord(e1, b->stream));
            BK(cudaEventSynchronize(e1));
            float ms = 0.0f;
            BK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms / kReps < best) {
                best = ms / kReps;
                best_s = s;
                best_c = cps;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    k_batch_clear_max<<<(b->n + 255) / 256, 256, 0, b->stream>>>(b->d_ctl, b->n);
    BK(cudaGetLastError());
    BK(cudaStreamSynchronize(b->stream));
    b->timing = timing;
    if (best_s < 0) return bfail(b, FVG_ERR_CUDA, "no tile shape's kernel could run");
    int rc = apply_schedule(b, best_s, best_c);
    if (rc) return rc;
    if (shape) *shape = best_s;
    if (ctas_per_sm) *ctas_per_sm = best_c;
    if (stage_ms) *stage_ms = best;
    return FVG_OK;
}

int fvg_batch_run(fvg_batch* b, double t_end, int max_steps, long long* cell_stages) {
    if (!b) return FVG_ERR_ARGUMENT;
    BK(cudaSetDevice(b->device));
    if (b->shape < 0) {
        int rc = fvg_batch_autotune(b, nullptr, nullptr, nullptr);
        if (rc) return rc;
    }
    k_batch_begin<<<(b->n + 255) / 256, 256, 0, b->stream>>>(b->d_ctl, b->n, t_end, max_steps);
    BK(cudaGetLastError());
    BK(enqueue_end(b, 0));
    // Steps are launched in chunks (a graph of graph_steps steps, or that many single launches when timing); the count of
    // running problems is copied back after each chunk and read one chunk late, so the GPU never waits for the host. A
    // chunk launched after every problem stopped finds an empty work list.
    if (!b->timing && !b->graph) {
        cudaGraph_t g;
        BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < b->graph_steps && e == cudaSuccess; ++k) e = enqueue_step(b);
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) return bfail(b, FVG_ERR_CUDA, "graph capture of the batch step failed");
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return bfail(b, FVG_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    cudaEvent_t ev[2];
    BK(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    BK(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    int rc = FVG_OK;
    for (long long k = 0;; ++k) {
        cudaError_t e = cudaSuccess;
        if (b->timing) {
            for (int s = 0; s < b->graph_steps && e == cudaSuccess; ++s) e = enqueue_step(b);
        } else {
            e = cudaGraphLaunch(b->graph, b->stream);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&b->h_remaining[k & 1], b->d_remaining, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[k & 1], b->stream);
        if (e == cudaSuccess && k > 0) e = cudaEventSynchronize(ev[(k - 1) & 1]);
        if (e != cudaSuccess) {
            rc = bfail(b, FVG_ERR_CUDA, std::string("batch step: ") + cudaGetErrorString(e));
            break;
        }
        if (b->timing) {   // timing: the chunk's events are read (and recycled) once it is done
            if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) {
                rc = bfail(b, FVG_ERR_CUDA, std::string("batch step: ") + cudaGetErrorString(e));
                break;
            }
            ev_flush(b);
        }
        if (k > 0 && b->h_remaining[(k - 1) & 1] == 0) break;
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (rc) return rc;
    BK(cudaStreamSynchronize(b->stream));
    if (b->timing) ev_flush(b);
    BK(cudaMemcpy(b->h_ctl.data(), b->d_ctl, sizeof(BatchCtl) * b->n, cudaMemcpyDeviceToHost));
    long long work = 0;
    bool diverged = false;
    for (int p = 0; p < b->n; ++p) {
        work += (long long)b->h_ctl[p].steps * b->nstages * (b->cell_off[p + 1] - b->cell_off[p]);
        diverged = diverged || b->h_ctl[p].status != 0;
    }
    if (cell_stages) *cell_stages = work;
    if (diverged) return bfail(b, FVG_ERR_DIVERGED, "a problem's solution diverged (non-finite wave speed or time step, or t no longer advances)");
    return FVG_OK;
}

int fvg_batch_problem(const fvg_batch* b, int i, double* t, int* steps, int* status) {
    if (!b || i < 0 || i >= b->n) return FVG_ERR_ARGUMENT;
    const BatchCtl& c = b->h_ctl[i];
    if (t) *t = c.t;
    if (steps) *steps = c.steps;
    if (status) *status = c.status;
    return FVG_OK;
}

int fvg_batch_stream(fvg_batch* b, void** stream) {
    if (!b || !stream) return FVG_ERR_ARGUMENT;
    *stream = b->stream;
    return FVG_OK;
}

int fvg_batch_set_timing(fvg_batch* b, int on) {
    if (!b) return FVG_ERR_ARGUMENT;
    b->timing = on != 0;
    b->t_ms = 0.0;
    b->t_n = 0;
    b->ev_used = 0;
    return FVG_OK;
}

int fvg_batch_get_timing(const fvg_batch* b, double* stage_ms, long long* stage_launches) {
    if (!b) return FVG_ERR_ARGUMENT;
    if (stage_ms) *stage_ms = b->t_ms;
    if (stage_launches) *stage_launches = b->t_n;
    return FVG_OK;
}

}   // extern "C"
