// The mixed-precision batched stage kernel (the mixed form of batch_stage_kernel; see mixed.cuh for what stays FP64).
// Built with --use_fast_math, as mixed.cu.
#include "batch.cuh"
#include "batch_api.h"
#include "mixed.cuh"

namespace fvg {
namespace {

// the thin y sweep of batch.cuh in the mixed form: the boundary-face states in FP64 (side_states), their primitives
// rounded to FP32, the Riemann solver and the balance in FP32 (as mixed_axis does for boundary faces)
template <int RIEMANN>
__device__ __forceinline__ float thin_face_mixed(const StageArgs& a, const Eos<float>& ef, float sb, int side, int i, St<float, 4>& F) {
    St<double, 4> UL, UR;
    side_states<4, false>(a.m, a.bc, a.eos, a.U, side, i, 0, 0, UL, UR);
    const St<double, 4> dl = c2p(a.eos, UL), dr = c2p(a.eos, UR);
    St<float, 4> wl, wr;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        wl[q] = (float)dl[q];
        wr[q] = (float)dr[q];
    }
    return face_flux_prim<RIEMANN>(ef, sb, wl, wr, 1, F);
}

template <int RIEMANN, int TX, int NT>
__device__ __forceinline__ void thin_y_mixed(const StageArgs& a, const Eos<float>& ef, float sb, float* __restrict__ acc, const int o3[3], float& smax) {
    const Mesh& m = a.m;
    const float A = (float)m.area[1];
    const bool same = copy_side(a.bc.type[2]) && copy_side(a.bc.type[3]);
    for (int c = threadIdx.x; c < TX; c += NT) {
        const int i = o3[0] + c;
        if (i >= m.nx) continue;
        St<float, 4> Fb, Ft;
        const float s_b = thin_face_mixed<RIEMANN>(a, ef, sb, 2, i, Fb);
        float s_t = s_b;
        if (same)
            Ft = Fb;
        else
            s_t = thin_face_mixed<RIEMANN>(a, ef, sb, 3, i, Ft);
        if (s_b > smax) smax = s_b;
        if (s_t > smax) smax = s_t;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            acc[q * TX + c] = __fmaf_rn(-(Ft[q] - Fb[q]), A, acc[q * TX + c]);   // (an explicit FMA, as mixed_axis's balance)
        }
    }
    __syncthreads();
}

template <int RECON, int RIEMANN, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) batch_mixed_kernel(const BatchArgs b) {
    using S = MixedShape<2, RECON, TX, TY, 1>;
    constexpr int NV = S::NV, NC = S::NC;
    extern __shared__ double smem_d[];
    double* red = smem_d;
    float* P = reinterpret_cast<float*>(smem_d + 32);
    float* WL = P + NV * S::EXT;
    float* WR = WL + NV * S::NF;
    float* acc = WR + NV * S::NF;
    unsigned char* Sf = reinterpret_cast<unsigned char*>(acc + NV * NC);
    __shared__ StageArgs sa;
    const int tid = threadIdx.x;
    const int nw = *b.nwork;
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        const BatchWork it = b.work[w];
        if (tid == 0) batch_item_args(b, b.prob[it.prob], sa);
        __syncthreads();
        const Mesh& m = sa.m;
        const Eos<float> ef{sa.eos.type, (float)sa.eos.gamma, (float)sa.eos.p_inf};
        const float sb = (float)sa.shock_blend, weps = (float)sa.weno_eps;
        const int tx = (m.nx + TX - 1) / TX;
        const int o3[3] = {(it.tile % tx) * TX, (it.tile / tx) * TY, 0};
        float smax = 0.0f;
        mixed_axis<0, 2, RECON, RIEMANN, TX, TY, 1, NT, false, false>(sa, ef, sb, weps, P, WL, WR, acc, Sf, o3, smax);
        bool thin = false;
        if constexpr (TY == 1) thin = thin_y(m, sa.bc);
        if (thin)
            thin_y_mixed<RIEMANN, TX, NT>(sa, ef, sb, acc, o3, smax);
        else
            mixed_axis<1, 2, RECON, RIEMANN, TX, TY, 1, NT, false, false>(sa, ef, sb, weps, P, WL, WR, acc, Sf, o3, smax);
        const double dt = b.ctl[it.prob].dt;
        for (int c = tid; c < NC; c += NT) {
            const int i = o3[0] + c % TX, j = o3[1] + c / TX;
            if (i >= m.nx || j >= m.ny) continue;
            const long long cell = (long long)j * m.nx + i;
            CellIn<NV> in;
            cell_load(sa, cell, in);
#pragma unroll
            for (int q = 0; q < NV; ++q) sa.out[q * m.plane + cell] = cell_out(sa, in, q, acc[q * NC + c], dt);
        }
        const double bm = block_max<NT>((double)smax, red);
        if (tid == 0) batch_stage_max(&b.ctl[it.prob], b.stage, bm);
        __syncthreads();
    }
}

template <int SHAPE, int RECON, int RIEMANN> struct MK {
    static constexpr BatchShape sh = kBatchShape[SHAPE];
    using S = MixedShape<2, RECON, sh.tx, sh.ty, 1>;
    static constexpr auto kern = batch_mixed_kernel<RECON, RIEMANN, sh.tx, sh.ty, sh.nt>;
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

template <int SHAPE, int RECON> BatchStage pick_r(int riemann) {
    return riemann == kLowMach ? MK<SHAPE, RECON, kLowMach>::get() : MK<SHAPE, RECON, kHLLC>::get();
}
template <int SHAPE> BatchStage pick_s(int recon, int riemann) {
    switch (recon) {
    case kMuscl: return pick_r<SHAPE, kMuscl>(riemann);
    case kWeno3: return pick_r<SHAPE, kWeno3>(riemann);
    default: return pick_r<SHAPE, kWeno5>(riemann);
    }
}

}   // namespace

BatchStage batch_mixed_stage(int shape, int recon, int riemann) {
    switch (shape) {
    case 0: return pick_s<0>(recon, riemann);
    case 1: return pick_s<1>(recon, riemann);
    case 2: return pick_s<2>(recon, riemann);
    default: return pick_s<3>(recon, riemann);
    }
}

}   // namespace fvg
