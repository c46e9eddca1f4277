// The troubled-cell sensor's kernels and their C ABI (include/fenice_gpu.h: fvg_sensor_*): training data from a run's
// state, the network's forward and backward passes on the tensor cores, the optimiser step, inference. Built with fast
// single-precision math, as the mixed-precision stage kernels that evaluate the network inside their tiles.
#include "../../include/fenice_gpu.h"
#include "grid.cuh"
#include "host_common.h"
#include "sensor.cuh"
#include "sensor_api.h"
#include "tc.cuh"
#include "tma.cuh"

#include <cuda_runtime.h>

using namespace fvg;

namespace {

// ------------------------------------------------------------------------------------------------ training data
__device__ __forceinline__ unsigned hash32(unsigned long long x, unsigned seed) {
    unsigned h = (unsigned)(x ^ (x >> 32)) * 0x9E3779B1u ^ seed * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    h *= 0x297A2D39u;
    h ^= h >> 15;
    return h;
}

// Features and label statistic of every (cell, axis) of a state. mode 0: all, at index cell * DIM + axis; mode 1: the
// troubled ones (statistic > tau) and every keep_div-th other one (by a hash), appended at an atomic counter up to cap.
// stats[0] += troubled, stats[1] += all. The statistic: the largest |WENO5-Z - linear| of the cell's two face values
// over the quantities, each relative to the quantity's physical scale at the cell (sensor_scale).
template <int DIM, int NV>
__global__ void k_sensor_extract(Mesh m, Bc bc, Eos<double> eos, const double* __restrict__ U, double weno_eps, int mode, int keep_div, unsigned seed,
                                 float tau, float* __restrict__ X, float* __restrict__ dep, int* count, long long cap,
                                 unsigned long long* stats) {
    const long long n = m.ncells * DIM;
    unsigned long long troubled = 0, total = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long c = e / DIM;
        const int axis = (int)(e % DIM);
        const int i = (int)(c % m.nx), j = (int)((c / m.nx) % m.ny), k = (int)(c / ((long long)m.nx * m.ny));
        double w5[5][NV];
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            const int d = s - 2;
            const St<double, NV> u = stencil_cons<DIM, NV>(m, bc, eos, U, i + (axis == 0 ? d : 0), j + (axis == 1 ? d : 0), k + (axis == 2 ? d : 0));
            const St<double, NV> w = c2p(eos, u);
#pragma unroll
            for (int q = 0; q < NV; ++q) w5[s][q] = w[q];
        }
        float f[kSensF];
        double D = 0.0;
        const double p_inf = eos.type == kIdeal ? 0.0 : eos.p_inf;
#pragma unroll
        for (int sq = 0; sq < kSensQ; ++sq) {
            const int var = sensor_var<NV>(sq, axis);
            const double scale = sensor_scale<double>(sq, w5[2][0], w5[2][3], eos.gamma, p_inf);
            float v[5];
#pragma unroll
            for (int s = 0; s < 5; ++s) v[s] = var >= 0 ? (float)w5[s][var < 0 ? 0 : var] : 0.0f;
            sensor_quantity_features(v, (float)scale, f + 5 * sq);
            if (var >= 0) {
                double cv[5];
#pragma unroll
                for (int s = 0; s < 5; ++s) cv[s] = w5[s][var];
                D = fmax(D, weno5z_face_gap(cv[0], cv[1], cv[2], cv[3], cv[4], weno_eps) / scale);
                D = fmax(D, weno5z_face_gap(cv[4], cv[3], cv[2], cv[1], cv[0], weno_eps) / scale);
            }
        }
        const bool bad = D > (double)tau;
        troubled += bad;
        total += 1;
        long long slot = e;
        if (mode == 1) {
            if (!bad && (keep_div <= 1 ? false : (hash32((unsigned long long)e, seed) % (unsigned)keep_div) != 0)) continue;
            slot = atomicAdd(count, 1);
            if (slot >= cap) continue;
        }
        float4* xo = reinterpret_cast<float4*>(X + slot * kSensK);
#pragma unroll
        for (int q = 0; q < kSensK / 4; ++q) {
            float4 v;
            v.x = 4 * q + 0 < kSensF ? f[4 * q + 0] : 0.0f;
            v.y = 4 * q + 1 < kSensF ? f[4 * q + 1] : 0.0f;
            v.z = 4 * q + 2 < kSensF ? f[4 * q + 2] : 0.0f;
            v.w = 4 * q + 3 < kSensF ? f[4 * q + 3] : 0.0f;
            xo[q] = v;
        }
        dep[slot] = (float)D;
    }
    if (stats) {
        atomicAdd(stats, troubled);
        atomicAdd(stats + 1, total);
    }
}

// ------------------------------------------------------------------------------------------------ training
// The device weights (bfloat16 copies, the transposed second layer) of float32 master parameters.
__device__ void pack_weights(const SensorP& P, SensorW* out) {
    for (int i = threadIdx.x; i < kSensH * kSensK; i += blockDim.x) out->W1[i] = __float2bfloat16_rn((i % kSensK) < kSensF ? P.W1[i] : 0.0f);
    for (int i = threadIdx.x; i < kSensH * kSensH; i += blockDim.x) {
        out->W2[i] = __float2bfloat16_rn(P.W2[i]);
        out->W2T[(i % kSensH) * kSensH + i / kSensH] = __float2bfloat16_rn(P.W2[i]);
    }
    for (int i = threadIdx.x; i < kSensH; i += blockDim.x) {
        out->b1[i] = P.b1[i];
        out->b2[i] = P.b2[i];
        out->w3[i] = round_bf16(P.w3[i]);
    }
    if (threadIdx.x == 0) out->b3 = P.b3;
}

__global__ void k_sensor_pack(const SensorP* P, SensorW* out) { pack_weights(*P, out); }

// One Adam step on the master parameters from grad (then cleared), and their device weights. One CTA.
__global__ void k_sensor_adam(float* P, float* m, float* v, float* grad, int step, float lr, float b1, float b2, float eps, SensorW* out) {
    const float c1 = 1.0f / (1.0f - powf(b1, (float)step)), c2 = 1.0f / (1.0f - powf(b2, (float)step));
    for (int i = threadIdx.x; i < kSensParams; i += blockDim.x) {
        const float gi = grad[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float p = P[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        if (i < kSensH * kSensK && (i % kSensK) >= kSensF) p = 0.0f;   // the padding inputs keep zero weights
        P[i] = p;
        grad[i] = 0.0f;
    }
    __syncthreads();
    pack_weights(*reinterpret_cast<const SensorP*>(P), out);
}

// ------------------------------------------------------------------------------------------------ the network on tcgen05
// A CTA of 256 threads evaluates the network 128 rows at a time on the fifth-generation tensor cores, as two independent
// warpgroups (warps 0-3 and 4-7) that take alternate tiles: each has its own tile X (128 x 32 bf16: the features, then the
// first layer's activations, which overwrite them once the first layer has read them) in shared memory in the MMA's
// canonical layout (tc.cuh), its own 32 TMEM columns for the layer's 128 x 32 f32
// accumulator, its own completion barrier and a named barrier for its 128 threads. The first thread of the group issues
// the two k-steps of a layer and commits them; the group's warps read the accumulator rows back (warp w its TMEM lane
// quarter w % 4: rows 32 (w % 4) .. + 31), add the bias, apply ReLU, round to bf16 and write X for the second layer, or,
// after the second layer, take the dot product with w3 in registers. The two groups' tiles interleave on the tensor core.
struct __align__(128) SensTc {
    // canonical, one per warpgroup: the features, then (once the first layer has read them) the first layer's activations
    __nv_bfloat16 X[2][128 * kSensK];
    __nv_bfloat16 W1[kSensH * kSensK];
    __nv_bfloat16 W2[kSensH * kSensH];
    float b1[kSensH], b2[kSensH], w3[kSensH];
    float b3;
    unsigned long long bar[2];
    uint32_t tmem;
    int fail;
};
constexpr int kTcPolls = 1 << 22;   // polls of a barrier before a wait gives up (a completion takes well under a microsecond)

__device__ __forceinline__ void wg_sync(int g) {   // the 128 threads of warpgroup g
    asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
}

// the weights into s (all threads), the barriers and 64 TMEM columns (warp 0); ends with a block barrier
__device__ __forceinline__ void sens_tc_setup(SensTc& s, const SensorW* __restrict__ wg) {
    for (int i = threadIdx.x; i < kSensH * kSensK; i += blockDim.x) {
        s.W1[tc::cl_index(i >> 5, i & 31)] = wg->W1[i];
        s.W2[tc::cl_index(i >> 5, i & 31)] = wg->W2[i];
    }
    for (int i = threadIdx.x; i < kSensH; i += blockDim.x) {
        s.b1[i] = wg->b1[i];
        s.b2[i] = wg->b2[i];
        s.w3[i] = wg->w3[i];
    }
    if (threadIdx.x == 0) {
        s.b3 = wg->b3;
        s.fail = 0;
        tma::mbar_init(&s.bar[0], 1);
        tma::mbar_init(&s.bar[1], 1);
        tma::fence_mbar_init();
    }
    if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(&s.tmem, 64);
    tma::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

__device__ __forceinline__ void sens_tc_release(SensTc& s) {
    tc::fence_before_sync();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(s.tmem, 64);
    }
}

// the next completion of warpgroup g's barrier (bounded; a wait that gives up sets s.fail)
__device__ __forceinline__ void sens_tc_wait(SensTc& s, int g, unsigned& phase) {
    int polls = 0;
    while (!tma::mbar_try_wait(&s.bar[g], phase & 1))
        if (++polls >= kTcPolls) {
            s.fail = 1;
            break;
        }
    ++phase;
    tc::fence_after_sync();
}

// The logit of row 32 (warp % 4) + lane of warpgroup g's feature tile s.X[g], which the group's threads have written (each
// fenced the async proxy after its writes); called by the 128 threads of the group, which it synchronises twice. phase
// counts the completions of the group's barrier so far.
__device__ __forceinline__ float sens_tc_tile(SensTc& s, int g, unsigned& phase) {
    const int q = (threadIdx.x >> 5) & 3, lane = threadIdx.x & 31;
    const bool issuer = (threadIdx.x & 127) == 0;
    constexpr uint32_t ID = tc::idesc_bf16<128, kSensH>();
    const uint32_t tcol = s.tmem + 32u * g, trow = tcol + ((uint32_t)(32 * q) << 16);
    tc::fence_before_sync();
    wg_sync(g);
    tc::fence_after_sync();
    if (issuer) {
        tc::mma_bf16(tcol, tc::smem_desc(s.X[g], 0), tc::smem_desc(s.W1, 0), ID, false);
        tc::mma_bf16(tcol, tc::smem_desc(s.X[g], 1), tc::smem_desc(s.W1, 1), ID, true);
        tc::commit(&s.bar[g]);
    }
    sens_tc_wait(s, g, phase);
    float d[32];
    tc::ld32(trow, d);
    const int r = 32 * q + lane;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        uint32_t pk[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int j = 8 * c + 2 * k;
            pk[k] = pack_bf16(fmaxf(d[j] + s.b1[j], 0.0f), fmaxf(d[j + 1] + s.b1[j + 1], 0.0f));
        }
        *reinterpret_cast<uint4*>(&s.X[g][tc::cl_index(r, 8 * c)]) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
    tma::fence_proxy_async();
    tc::fence_before_sync();
    wg_sync(g);
    tc::fence_after_sync();
    if (issuer) {
        tc::mma_bf16(tcol, tc::smem_desc(s.X[g], 0), tc::smem_desc(s.W2, 0), ID, false);
        tc::mma_bf16(tcol, tc::smem_desc(s.X[g], 1), tc::smem_desc(s.W2, 1), ID, true);
        tc::commit(&s.bar[g]);
    }
    sens_tc_wait(s, g, phase);
    tc::ld32(trow, d);
    float z = 0.0f;
#pragma unroll
    for (int j = 0; j < kSensH; ++j) z += round_bf16(fmaxf(d[j] + s.b2[j], 0.0f)) * s.w3[j];
    return z + s.b3;
}

// ---- training on tcgen05
// Gradients of the mean class-weighted binary cross-entropy (weight wpos on troubled samples) over n samples, added to
// grad (a SensorP of float32) and the loss sum to *loss. A CTA of 256 threads takes 128 samples at a time; every product is
// a tcgen05.mma with bf16 operands in shared memory and f32 accumulators in TMEM:
//   forward   z1 = x W1^T, z2 = h1 W2^T                                      (M = 128 samples, N = 32, K = 32)
//   backward  dh1 = dh2 W2 (masked by z1 > 0)                                (M = 128, N = 32, K = 32)
//   weights   G += A^T B over the samples, accumulated in TMEM over all the CTA's tiles (M = 128, N = 96, K = 128 per tile)
//             with A = [dh2 | dh1 | dz | 0] (128 columns) and B = [h1 | x | h2] (96 columns; x's padding input 31 set to 1):
//             G[0:32, 0:32] = dW2, G[0:32, 63] = db2, G[32:64, 32:64] = dW1 (column 63: db1), G[64, 64:96] = dw3, G[64, 63] = db3.
// A and B are stored as samples x columns in the canonical layout (core matrices of 8 samples x 8 columns, 128 bytes, the
// column groups of an 8-sample group adjacent): read with the samples as K they are MN-major operands, with the samples as
// M K-major ones. Back-propagated values enter the products rounded to bf16 (dh2, dh1, dz).
constexpr int kGA = 128, kGB = 96;   // columns of the A and B tiles
struct __align__(1024) GradTc {
    __nv_bfloat16 A[128 * kGA];   // 16 column groups per 8-sample group (2048 bytes)
    __nv_bfloat16 B[128 * kGB];   // 12 column groups per 8-sample group (1536 bytes)
    __nv_bfloat16 W1[kSensH * kSensK], W2[kSensH * kSensH], W2T[kSensH * kSensH];   // canonical, K-major
    float b1[kSensH], b2[kSensH], w3[kSensH];
    float b3, loss;
    unsigned long long bar;
    uint32_t tmem;
    int fail;
};
constexpr int kGradSmem = (int)sizeof(GradTc);

// element offset of (sample r, column c) of a canonical tile with `groups` column groups
__device__ __forceinline__ int gt_index(int r, int c, int groups) { return ((r >> 3) * groups + (c >> 3)) * 64 + (r & 7) * 8 + (c & 7); }

// the next completion of the barrier, waited for by warps 0-3 (bounded: a wait that gives up sets s.fail)
__device__ __forceinline__ void grad_wait(GradTc& s, unsigned& phase) {
    int polls = 0;
    while (!tma::mbar_try_wait(&s.bar, phase & 1))
        if (++polls >= kTcPolls) {
            s.fail = 1;
            break;
        }
    ++phase;
    tc::fence_after_sync();
}

// every thread's shared-memory writes visible to the next MMA, every TMEM read done before it
__device__ __forceinline__ void grad_sync() {
    tma::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

__global__ void __launch_bounds__(256) k_sensor_grad(const SensorW* __restrict__ wg, const float* __restrict__ X, const float* __restrict__ y, long long n,
                                                     float wpos, float inv_n, float* __restrict__ grad, float* __restrict__ loss) {
    extern __shared__ __align__(1024) unsigned char gsm[];
    GradTc& s = *reinterpret_cast<GradTc*>(gsm);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kSensH * kSensK; i += blockDim.x) {
        s.W1[tc::cl_index(i >> 5, i & 31)] = wg->W1[i];
        s.W2[tc::cl_index(i >> 5, i & 31)] = wg->W2[i];
        s.W2T[tc::cl_index(i >> 5, i & 31)] = wg->W2T[i];
    }
    for (int i = threadIdx.x; i < kSensH; i += blockDim.x) {
        s.b1[i] = wg->b1[i];
        s.b2[i] = wg->b2[i];
        s.w3[i] = wg->w3[i];
    }
    for (int i = threadIdx.x; i < 128 * kGA; i += blockDim.x) s.A[i] = __float2bfloat16_rn(0.0f);   // columns 65 .. 127 stay 0
    if (threadIdx.x == 0) {
        s.b3 = wg->b3;
        s.loss = 0.0f;
        s.fail = 0;
        tma::mbar_init(&s.bar, 1);
        tma::fence_mbar_init();
    }
    if (warp == 0) tc::tmem_alloc(&s.tmem, 128);   // columns 0-95: G; 96-127: the layers' accumulator
    grad_sync();
    const uint32_t tG = s.tmem, tZ = s.tmem + 96, lane_off = (uint32_t)(32 * (warp & 3)) << 16;
    constexpr uint32_t ID32 = tc::idesc_bf16<128, 32>(), IDG = tc::idesc_bf16<128, kGB, true>();
    // tZ = A W^T of a 128 x 32 block of a tile read K-major (samples as M: 8-sample groups `sbo` bytes apart, column groups
    // 128), committed to the barrier
    auto layer = [&](const void* abase, uint32_t aoff, uint32_t sbo, const __nv_bfloat16* W) {
        if (threadIdx.x == 0) {
            tc::mma_bf16(tZ, tc::smem_desc_at(abase, aoff, 128, sbo), tc::smem_desc(W, 0), ID32, false);
            tc::mma_bf16(tZ, tc::smem_desc_at(abase, aoff + 256, 128, sbo), tc::smem_desc(W, 1), ID32, true);
            tc::commit(&s.bar);
        }
    };
    unsigned phase = 0;
    float lsum = 0.0f;
    const long long ntile = (n + 127) / 128;
    int done = 0;
    for (long long tt = blockIdx.x; tt < ntile; tt += gridDim.x, ++done) {
        const long long r0 = tt * 128;
        // x into B's columns 32 .. 63 (input 31 = 1 on a sample: the bias column of the products)
        for (int idx = threadIdx.x; idx < 128 * kSensK; idx += blockDim.x) {
            const int r = idx / kSensK, c = idx % kSensK;
            const bool in = r0 + r < n;
            const float v = !in ? 0.0f : (c < kSensF ? X[(r0 + r) * kSensK + c] : (c == kSensK - 1 ? 1.0f : 0.0f));
            s.B[gt_index(r, 32 + c, 12)] = __float2bfloat16_rn(v);
        }
        grad_sync();
        layer(s.B, 4 * 128, 1536, s.W1);   // z1 = x W1^T
        uint32_t mask1 = 0;
        if (warp < 4) {
            grad_wait(s, phase);
            float d[32];
            tc::ld32(tZ + lane_off, d);
            const int r = 32 * warp + lane;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const float z = d[j] + s.b1[j];
                mask1 |= (z > 0.0f ? 1u : 0u) << j;
                s.B[gt_index(r, j, 12)] = __float2bfloat16_rn(fmaxf(z, 0.0f));
            }
        }
        grad_sync();
        layer(s.B, 0, 1536, s.W2);   // z2 = h1 W2^T
        if (warp < 4) {
            grad_wait(s, phase);
            float d[32];
            tc::ld32(tZ + lane_off, d);
            const int r = 32 * warp + lane;
            const long long gr = r0 + r;
            float h2[32], zsum = 0.0f;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                h2[j] = round_bf16(fmaxf(d[j] + s.b2[j], 0.0f));
                zsum += h2[j] * s.w3[j];
            }
            const float z = zsum + s.b3;
            float dz = 0.0f;
            if (gr < n) {
                const float yv = y[gr], wv = yv > 0.5f ? wpos : 1.0f;
                lsum += wv * (fmaxf(z, 0.0f) + log1pf(__expf(-fabsf(z))) - yv * z);
                dz = wv * (1.0f / (1.0f + __expf(-z)) - yv) * inv_n;
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                s.A[gt_index(r, j, 16)] = __float2bfloat16_rn(d[j] + s.b2[j] > 0.0f ? dz * s.w3[j] : 0.0f);
                s.B[gt_index(r, 64 + j, 12)] = __float2bfloat16_rn(h2[j]);
            }
            s.A[gt_index(r, 64, 16)] = __float2bfloat16_rn(dz);
        }
        grad_sync();
        layer(s.A, 0, 2048, s.W2T);   // dh2 W2 (W2T: [in][out], read K-major)
        if (warp < 4) {
            grad_wait(s, phase);
            float d[32];
            tc::ld32(tZ + lane_off, d);
            const int r = 32 * warp + lane;
#pragma unroll
            for (int j = 0; j < 32; ++j) s.A[gt_index(r, 32 + j, 16)] = __float2bfloat16_rn((mask1 >> j) & 1u ? d[j] : 0.0f);
        }
        grad_sync();
        // G += A^T B over the tile's 128 samples: 8 k-steps of 16 samples (two 8-sample groups each)
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < 8; ++k)
                tc::mma_bf16(tG, tc::smem_desc_at(s.A, 4096u * k, 2048, 128), tc::smem_desc_at(s.B, 3072u * k, 1536, 128), IDG, done > 0 || k > 0);
            tc::commit(&s.bar);
        }
        if (warp < 4) grad_wait(s, phase);   // the tiles are rewritten next: the products must have read them
        grad_sync();
    }
    // ---- the CTA's sums into grad (warps 0-3: TMEM lane m = 32 warp + lane holds row m of G)
    if (warp < 4 && done > 0 && !s.fail) {
        SensorP& G = *reinterpret_cast<SensorP*>(grad);
        const int m = 32 * warp + lane;
        float g0[32], g1[32], g2[32];
        tc::ld32(tG + lane_off, g0);
        tc::ld32(tG + lane_off + 32, g1);
        tc::ld32(tG + lane_off + 64, g2);
        if (m < 32) {
#pragma unroll
            for (int i = 0; i < 32; ++i) atomicAdd(&G.W2[m * kSensH + i], g0[i]);
            atomicAdd(&G.b2[m], g1[31]);
        } else if (m < 64) {
#pragma unroll
            for (int i = 0; i < kSensF; ++i) atomicAdd(&G.W1[(m - 32) * kSensK + i], g1[i]);
            atomicAdd(&G.b1[m - 32], g1[31]);
        } else if (m == 64) {
#pragma unroll
            for (int j = 0; j < 32; ++j) atomicAdd(&G.w3[j], g2[j]);
            atomicAdd(&G.b3, g1[31]);
        }
    }
    // the loss: lanes, then warps, then the CTA (NaN when a wait gave up)
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, k);
    if (lane == 0 && warp < 4) atomicAdd(&s.loss, lsum);
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(loss, s.fail ? __int_as_float(0x7fc00000) : s.loss);
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(s.tmem, 128);
    }
}

// Logits of n feature rows, 128 rows per tile on the tensor cores (a NaN logit: a tensor-core step did not complete):
// warpgroup g of CTA b takes tiles 2 b + g, 2 b + g + 2 gridDim.x, ...
__global__ void __launch_bounds__(256) k_sensor_infer(const SensorW* __restrict__ wg, const float* __restrict__ X, long long n, float* __restrict__ logits) {
    __shared__ SensTc st;
    sens_tc_setup(st, wg);
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    unsigned phase = 0;
    const long long ntile = (n + 127) / 128;
    for (long long tt = 2LL * blockIdx.x + g; tt < ntile; tt += 2LL * gridDim.x) {
        const long long r0 = tt * 128;
        // row r, column group c: two float4 loads, one 16-byte store of 8 bf16 into the canonical tile
        for (int idx = t; idx < 128 * 4; idx += 128) {
            const int r = idx >> 2, c = idx & 3;
            uint32_t pk[4] = {0u, 0u, 0u, 0u};
            if (r0 + r < n && 8 * c < kSensF) {
                const float4 a = *reinterpret_cast<const float4*>(X + (r0 + r) * kSensK + 8 * c);
                const float4 b = *reinterpret_cast<const float4*>(X + (r0 + r) * kSensK + 8 * c + 4);
                const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int j = 8 * c + 2 * k;
                    pk[k] = pack_bf16(j < kSensF ? v[2 * k] : 0.0f, j + 1 < kSensF ? v[2 * k + 1] : 0.0f);
                }
            }
            *reinterpret_cast<uint4*>(&st.X[g][tc::cl_index(r, 8 * c)]) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        tma::fence_proxy_async();
        const float z = sens_tc_tile(st, g, phase);
        const int r = 32 * ((threadIdx.x >> 5) & 3) + (threadIdx.x & 31);
        if (r0 + r < n) logits[r0 + r] = st.fail ? __int_as_float(0x7fc00000) : z;
    }
    sens_tc_release(st);
}

// ------------------------------------------------------------------------------------------------ the gate
__device__ __forceinline__ bool refresh_due(const Ctl* ctl, int every) { return !ctl || (ctl->active && ctl->steps % every == 0); }

// The network's flags of every (cell, axis), tiled: a CTA takes a BX x BY (x BZ) block of cells, recovers the
// primitive state of the block and a 2-cell halo once per cell into shared memory (float), then its warps take 16
// (cell, axis) rows at a time: features of the row's 5-cell stencil into the warp's bf16 tile (one lane per row and
// quantity), logits on the tensor cores.
template <int DIM, int NV, int BX, int BY, int BZ>
__global__ void __launch_bounds__(256) k_sensor_flags_t(Mesh m, Bc bc, Eos<double> eos, const double* __restrict__ U, const SensorW* __restrict__ wg,
                                                        float theta, unsigned char* __restrict__ flags, const Ctl* ctl, int every, int nb0, int nb1,
                                                        int* err) {
    if (!refresh_due(ctl, every)) return;
    constexpr int EX = BX + 4, EY = BY + 4, EZ = DIM == 3 ? BZ + 4 : 1, BOX = EX * EY * EZ, NC = BX * BY * BZ, ROWS = NC * DIM;
    // the planes of the primitive variables PS floats apart, PS = 7 (mod 32): the lanes that read the five quantities of
    // one stencil position read five different banks (a plane stride that is a multiple of 32 puts them on one)
    constexpr int PS = BOX + ((7 - BOX % 32) + 32) % 32;
    extern __shared__ __align__(1024) unsigned char fsm[];   // SensTc, then the primitive planes P (flags_smem bytes)
    SensTc& st = *reinterpret_cast<SensTc*>(fsm);
    float* P = reinterpret_cast<float*>(fsm + sizeof(SensTc));
    sens_tc_setup(st, wg);
    const int b = blockIdx.x;
    const int o0 = (b % nb0) * BX, o1 = ((b / nb0) % nb1) * BY, o2 = DIM == 3 ? (b / (nb0 * nb1)) * BZ : 0;
    for (int e = threadIdx.x; e < BOX; e += blockDim.x) {
        const int i = o0 + e % EX - 2, j = o1 + (e / EX) % EY - 2, k = DIM == 3 ? o2 + e / (EX * EY) - 2 : 0;
        const St<double, NV> wv = c2p(eos, stencil_cons<DIM, NV>(m, bc, eos, U, i, j, k));
#pragma unroll
        for (int q = 0; q < NV; ++q) P[q * PS + e] = (float)wv[q];
    }
    __syncthreads();
    const int g = threadIdx.x >> 7, q = (threadIdx.x >> 5) & 3, lane = threadIdx.x & 31;
    const float gam = (float)eos.gamma, pinf = eos.type == kIdeal ? 0.0f : (float)eos.p_inf;
    unsigned phase = 0;
    // warpgroup g takes the 128-row tiles 2 k + g of the block's ROWS (cell, axis) rows
    for (int t0 = 128 * g; t0 < ROWS; t0 += 256) {
        // features of the tile's rows: warp q of the group rows 32 q .. 32 q + 31, one lane per (row, quantity)
        for (int it = lane; it < 32 * kSensQ; it += 32) {
            const int row = 32 * q + it / kSensQ, sq = it % kSensQ, r = t0 + row;
            float f[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            if (r < ROWS) {
                const int c = r / DIM, axis = r % DIM;
                const int var = sensor_var<NV>(sq, axis);
                if (var >= 0) {
                    const int e = ((DIM == 3 ? c / (BX * BY) + 2 : 0) * EY + (c / BX) % BY + 2) * EX + c % BX + 2;
                    const int st_ = axis == 0 ? 1 : (axis == 1 ? EX : EX * EY);
                    float v[5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) v[k] = P[var * PS + e + (k - 2) * st_];
                    sensor_quantity_features(v, sensor_scale<float>(sq, P[e], P[3 * PS + e], gam, pinf), f);
                }
            }
#pragma unroll
            for (int k = 0; k < 5; ++k) st.X[g][tc::cl_index(row, 5 * sq + k)] = __float2bfloat16_rn(f[k]);
        }
        // the padding inputs (the previous tile's hidden values sit there)
        for (int k = kSensF; k < kSensK; ++k) st.X[g][tc::cl_index(threadIdx.x & 127, k)] = __float2bfloat16_rn(0.0f);
        tma::fence_proxy_async();
        const float z = sens_tc_tile(st, g, phase);
        const int r = t0 + 32 * q + lane;
        if (r < ROWS) {
            const int c = r / DIM, axis = r % DIM;
            const int i = o0 + c % BX, j = o1 + (c / BX) % BY, k = DIM == 3 ? o2 + c / (BX * BY) : 0;
            // a tensor-core step that did not complete leaves the row WENO5-Z
            if (i < m.nx && j < m.ny && k < m.nz) flags[axis * m.plane + ((long long)k * m.ny + j) * m.nx + i] = (!st.fail && z < theta) ? 0 : 1;
        }
    }
    if (st.fail && threadIdx.x == 0 && err) atomicExch(err, 6);
    sens_tc_release(st);
}

// The tile flags of the stage kernels from the network's flags. Tile b is linear along axis a (0) when no cell whose
// reconstructions along a it needs (the tile extended by one cell along a) has a flagged (cell, a) pair within `radius`
// cells per axis (the distance a wave travels until the next refresh): a max filter of that radius followed by the OR over
// the extended tile is the OR over one box, the tile extended by radius + 1 cells along a and radius along the other axes,
// each range wrapped across a periodic pair of sides and clipped at the others. A tile whose extension along a leaves the
// mesh across a side that is not periodic stays WENO5-Z. The box is taken in two passes: k_gate_rows ORs every row of
// cells over each tile column's x range, k_gate_tiles ORs those bytes over the tile's y and z ranges. On a part of a
// decomposed mesh (split >= 0) a tile whose box reaches an interface of the part along the split axis (radius + 1 cells)
// stays WENO5-Z along every axis: the neighbour's flags are not held here, and both parts then solve an interface face alike.
__device__ __forceinline__ int wrap_index(int q, int n) { return q >= 0 && q < n ? q : ((q % n) + n) % n; }

// the box's range along axis d for a tile starting at o (inclusive; beyond a periodic side the indices wrap when read)
__device__ __forceinline__ void gate_range(int o, int T, int n, int d, int a, int radius, bool periodic, int& lo, int& hi) {
    lo = o;
    hi = o + T - 1 < n - 1 ? o + T - 1 : n - 1;
    if (d == a) {
        lo -= 1;
        hi += 1;
    }
    lo -= radius;
    hi += radius;
    if (!periodic) {
        lo = lo < 0 ? 0 : lo;
        hi = hi > n - 1 ? n - 1 : hi;
    }
}

// rows[(a * nz + z) * ny + y][t0] = OR of flags[a] over the row (y, z) and the x range of tile column t0
template <int DIM>
__global__ void k_gate_rows(Mesh m, const unsigned char* __restrict__ flags, int TX, int t0n, int per0, int radius, unsigned char* __restrict__ rows,
                            const Ctl* ctl, int every) {
    if (!refresh_due(ctl, every)) return;
    const long long total = (long long)DIM * m.nz * m.ny * t0n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int t0 = (int)(e % t0n);
        const long long ry = e / t0n;                           // (a * nz + z) * ny + y
        const int a = (int)(ry / ((long long)m.nz * m.ny));
        const unsigned char* row = flags + a * m.plane + (ry - (long long)a * m.nz * m.ny) * m.nx;
        int lo, hi;
        gate_range(t0 * TX, TX, m.nx, 0, a, radius, per0 != 0, lo, hi);
        bool f = false;
        for (int x = lo; x <= hi; ++x) f |= row[wrap_index(x, m.nx)] != 0;
        rows[e] = f ? 1 : 0;
    }
}

// out[a * ntiles + b] from the row bytes over the tile's y and z ranges, the edge rule; counts += [linear, all]
template <int DIM>
__global__ void k_gate_tiles(Mesh m, const unsigned char* __restrict__ rows, int TX, int TY, int TZ, int t0n, int t1n, int t2n, int per0, int per1,
                             int per2, int radius, unsigned char* __restrict__ out, const Ctl* ctl, int every, unsigned long long* counts, int split,
                             int peer_lo, int peer_hi) {
    if (!refresh_due(ctl, every)) return;
    const long long ntiles = (long long)t0n * t1n * t2n, total = DIM * ntiles;
    const int n3[3] = {m.nx, m.ny, m.nz}, per[3] = {per0, per1, per2};
    unsigned long long lin = 0, all = 0;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(w / ntiles);
        const long long b = w % ntiles;
        const int t0 = (int)(b % t0n), t1 = (int)((b / t0n) % t1n), t2 = (int)(b / ((long long)t0n * t1n));
        const int o[3] = {t0 * TX, t1 * TY, t2 * TZ};
        // the extension along a leaves the mesh across a side that is not periodic
        const int T3[3] = {TX, TY, TZ};
        const int ha = o[a] + T3[a] - 1 < n3[a] - 1 ? o[a] + T3[a] - 1 : n3[a] - 1;
        bool any = !per[a] && (o[a] - 1 < 0 || ha + 1 > n3[a] - 1);
        if (split >= 0) {   // the box reaches an interface of this part
            const int hs = o[split] + T3[split] - 1 < n3[split] - 1 ? o[split] + T3[split] - 1 : n3[split] - 1;
            any = any || (peer_lo && o[split] - (radius + 1) < 0) || (peer_hi && hs + radius + 1 > n3[split] - 1);
        }
        int lo1, hi1, lo2 = 0, hi2 = 0;
        gate_range(o[1], TY, n3[1], 1, a, radius, per[1] != 0, lo1, hi1);
        if (DIM == 3) gate_range(o[2], TZ, n3[2], 2, a, radius, per[2] != 0, lo2, hi2);
        const unsigned char* src = rows + (long long)a * m.nz * m.ny * t0n + t0;
        for (int z = lo2; z <= hi2 && !any; ++z) {
            const long long zo = (long long)wrap_index(z, n3[2]) * m.ny;
            for (int y = lo1; y <= hi1; ++y) any |= src[(zo + wrap_index(y, n3[1])) * t0n] != 0;
        }
        out[w] = any ? 1 : 0;
        lin += any ? 0 : 1;
        all += 1;
    }
    if (counts) {
#pragma unroll
        for (int k = 16; k > 0; k >>= 1) {
            lin += __shfl_xor_sync(0xffffffffu, lin, k);
            all += __shfl_xor_sync(0xffffffffu, all, k);
        }
        if ((threadIdx.x & 31) == 0 && all) {
            atomicAdd(counts, lin);
            atomicAdd(counts + 1, all);
        }
    }
}

int grid_for(long long rows) {
    const long long chunks = (rows + 15) / 16, b = (chunks + 7) / 8;
    return (int)(b < 1 ? 1 : (b > 148 * 4 ? 148 * 4 : b));
}

// the dynamic shared memory of k_sensor_flags_t<DIM, NV, BX, BY, BZ>: the network's tiles, then NV primitive planes of the
// block and its 2-cell halo (plane stride 7 mod 32)
template <int DIM, int NV, int BX, int BY, int BZ> constexpr int flags_smem() {
    constexpr int BOX = (BX + 4) * (BY + 4) * (DIM == 3 ? BZ + 4 : 1);
    return (int)sizeof(SensTc) + 4 * NV * (BOX + ((7 - BOX % 32) + 32) % 32);
}

template <int DIM, int NV, int BX, int BY, int BZ>
cudaError_t launch_flags(int blocks, cudaStream_t s, const Mesh& m, const Bc& bc, const Eos<double>& eos, const double* U, const SensorW* w, float theta,
                         unsigned char* flags0, const Ctl* ctl, int every, int b0, int b1, int* err) {
    constexpr int SM = flags_smem<DIM, NV, BX, BY, BZ>();
    static const cudaError_t attr = cudaFuncSetAttribute(k_sensor_flags_t<DIM, NV, BX, BY, BZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
    if (attr != cudaSuccess) return attr;
    k_sensor_flags_t<DIM, NV, BX, BY, BZ><<<blocks, 256, SM, s>>>(m, bc, eos, U, w, theta, flags0, ctl, every, b0, b1, err);
    return cudaGetLastError();
}

}   // namespace

cudaError_t fvg::sensor_refresh(const Mesh& m, const Bc& bc, const Eos<double>& eos, int dim, const double* U, const void* weights, float theta,
                                int radius, const int periodic[3], unsigned char* flags0, unsigned char* rows, const int tile[3],
                                const int tiles[3], unsigned char* tile_flags, const Ctl* ctl, int every, unsigned long long* counts,
                                cudaStream_t s, int split, int peer_lo, int peer_hi) {
    const SensorW* w = static_cast<const SensorW*>(weights);
    // a tensor-core step of the network that did not complete: status 6 in the run's control block
    int* err = ctl ? const_cast<int*>(&ctl->status) : nullptr;
    if (dim == 3) {
        const int b0 = (m.nx + 7) / 8, b1 = (m.ny + 7) / 8, b2 = (m.nz + 3) / 4;
        const cudaError_t e = launch_flags<3, 5, 8, 8, 4>(b0 * b1 * b2, s, m, bc, eos, U, w, theta, flags0, ctl, every, b0, b1, err);
        if (e != cudaSuccess) return e;
    } else {
        const int b0 = (m.nx + 31) / 32, b1 = (m.ny + 7) / 8;
        const cudaError_t e = launch_flags<2, 4, 32, 8, 1>(b0 * b1, s, m, bc, eos, U, w, theta, flags0, ctl, every, b0, b1, err);
        if (e != cudaSuccess) return e;
    }
    const long long nr = (long long)dim * m.nz * m.ny * tiles[0];
    const int rb = (int)((nr + 255) / 256 < 148 * 16 ? (nr + 255) / 256 : 148 * 16);
    const long long nt = (long long)tiles[0] * tiles[1] * tiles[2] * dim;
    const int tb = (int)((nt + 255) / 256 < 148 * 16 ? (nt + 255) / 256 : 148 * 16);
    if (dim == 3) {
        k_gate_rows<3><<<rb, 256, 0, s>>>(m, flags0, tile[0], tiles[0], periodic[0], radius, rows, ctl, every);
        k_gate_tiles<3><<<tb, 256, 0, s>>>(m, rows, tile[0], tile[1], tile[2], tiles[0], tiles[1], tiles[2], periodic[0], periodic[1], periodic[2], radius,
                                           tile_flags, ctl, every, counts, split, peer_lo, peer_hi);
    } else {
        k_gate_rows<2><<<rb, 256, 0, s>>>(m, flags0, tile[0], tiles[0], periodic[0], radius, rows, ctl, every);
        k_gate_tiles<2><<<tb, 256, 0, s>>>(m, rows, tile[0], tile[1], 1, tiles[0], tiles[1], 1, periodic[0], periodic[1], 0, radius, tile_flags, ctl,
                                           every, counts, split, peer_lo, peer_hi);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------ C ABI
namespace {
int serr(int code, const char* msg) {
    *create_error_slot() = msg;
    return code;
}
#define SK(call)                                                                                \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) return serr(FVG_ERR_CUDA, cudaGetErrorString(e_));               \
    } while (0)
}   // namespace

extern "C" {

int fvg_sensor_sizes(int* n_params, int* weights_bytes, int* n_inputs) {
    if (n_params) *n_params = kSensParams;
    if (weights_bytes) *weights_bytes = (int)sizeof(SensorW);
    if (n_inputs) *n_inputs = kSensK;
    return FVG_OK;
}

int fvg_sensor_extract(fvg_run* run, int mode, int keep_div, unsigned seed, float tau, float* X, float* departure, int* count, long long capacity,
                       unsigned long long* stats) {
    RunView v;
    if (!run_view(run, &v) || !X || !departure || (mode == 1 && !count)) return serr(FVG_ERR_ARGUMENT, "null argument");
    if (mode != 0 && mode != 1) return serr(FVG_ERR_ARGUMENT, "mode must be 0 (all) or 1 (sampled)");
    if (mode == 0 && capacity < v.m.ncells * v.dim) return serr(FVG_ERR_ARGUMENT, "capacity below cells x axes");
    SK(cudaSetDevice(v.device));
    const long long n = v.m.ncells * v.dim;
    const int blocks = (int)((n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8);
    if (v.dim == 3)
        k_sensor_extract<3, 5><<<blocks, 256, 0, v.stream>>>(v.m, v.bc, v.eos, v.U, v.weno_eps, mode, keep_div, seed, tau, X, departure, count, capacity, stats);
    else
        k_sensor_extract<2, 4><<<blocks, 256, 0, v.stream>>>(v.m, v.bc, v.eos, v.U, v.weno_eps, mode, keep_div, seed, tau, X, departure, count, capacity, stats);
    SK(cudaGetLastError());
    SK(cudaStreamSynchronize(v.stream));
    return FVG_OK;
}

int fvg_sensor_grad(const void* weights, const float* X, const float* y, long long n, float wpos, float* grad, float* loss, void* stream) {
    if (!weights || !X || !y || !grad || !loss || n < 1) return serr(FVG_ERR_ARGUMENT, "null argument or no samples");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static const cudaError_t attr = cudaFuncSetAttribute(k_sensor_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, kGradSmem);
    SK(attr);
    k_sensor_grad<<<grid_for(n), 256, kGradSmem, s>>>(static_cast<const SensorW*>(weights), X, y, n, wpos, 1.0f / (float)n, grad, loss);
    SK(cudaGetLastError());
    return FVG_OK;
}

int fvg_sensor_adam(float* params, float* m, float* v, float* grad, int step, float lr, float beta1, float beta2, float eps, void* weights, void* stream) {
    if (!params || !m || !v || !grad || !weights || step < 1) return serr(FVG_ERR_ARGUMENT, "null argument or step < 1");
    k_sensor_adam<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(params, m, v, grad, step, lr, beta1, beta2, eps, static_cast<SensorW*>(weights));
    SK(cudaGetLastError());
    return FVG_OK;
}

int fvg_sensor_pack(const float* params, void* weights, void* stream) {
    if (!params || !weights) return serr(FVG_ERR_ARGUMENT, "null argument");
    k_sensor_pack<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const SensorP*>(params), static_cast<SensorW*>(weights));
    SK(cudaGetLastError());
    return FVG_OK;
}

int fvg_sensor_infer(const void* weights, const float* X, long long n, float* logits, void* stream) {
    if (!weights || !X || !logits || n < 1) return serr(FVG_ERR_ARGUMENT, "null argument or no samples");
    k_sensor_infer<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const SensorW*>(weights), X, n, logits);
    SK(cudaGetLastError());
    return FVG_OK;
}

}   // extern "C"
