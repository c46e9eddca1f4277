// The learned troubled-cell sensor: a small MLP that reads a cell's 5-cell stencil along a sweep axis and decides whether
// the cell's two WENO5-Z reconstructions along that axis may take the linear fifth-order upwind values instead.
//
// Inputs (per cell and axis): the 5 cells c-2 .. c+2 along the axis, 5 primitive quantities each (rho, the normal
// velocity, the two tangential velocities (the second is 0 on a 2-D mesh), p). Per quantity: the stencil's shape (the
// four differences v_k - v0 over the largest of them) and its amplitude (log2(1 + 1e4 M / s) / 4, M that largest
// difference, s the quantity's physical scale at the cell: rho for the density, the sound speed for the velocities,
// p + p_inf for the pressure). 25 features, padded with zeros to the 32 of two tensor-core k-steps.
// Network: 32 -> 32 (ReLU) -> 32 (ReLU) -> 1 logit; weights and hidden activations in bfloat16, sums in float32 (the
// dense layers as tcgen05 MMAs of 128 rows with f32 accumulators in tensor memory: sensor.cu, tc.cuh). The cell is smooth (linear reconstruction)
// when the logit is below a threshold chosen for a low miss rate; otherwise, and for every cell the network is not sure
// about, WENO5-Z stays.
// Label (what the network learns): the largest gap |WENO5-Z - linear| between the cell's two WENO5-Z face values (the
// reference's weno5z, cpp/src/Schemes.cpp:328-353) and the linear fifth-order upwind values there, over the quantities,
// relative to the quantity's physical scale, above a label threshold: what the linear reconstruction would change at the
// cell's faces. (WENO-Z weights that depart from the linear ones at a smooth extremum or where a velocity crosses zero
// change the face values by a negligible amount, and such cells pass.)
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace fvg {

constexpr int kSensQ = 5;             // quantities per stencil cell
constexpr int kSensF = 5 * kSensQ;    // features
constexpr int kSensK = 32;            // padded input width
constexpr int kSensH = 32;            // hidden width

// Device weights of the network as the kernels read them.
struct SensorW {
    __nv_bfloat16 W1[kSensH * kSensK];    // [out][in], inputs kSensF .. kSensK-1 zero
    __nv_bfloat16 W2[kSensH * kSensH];    // [out][in]
    float b1[kSensH], b2[kSensH];
    float w3[kSensH];                     // bfloat16-rounded
    float b3;
    float pad[3];
    __nv_bfloat16 W2T[kSensH * kSensH];   // [in][out] (the backward pass's operand; inference copies what precedes it)
};
constexpr int kSensInferBytes = 2 * kSensH * kSensK + 2 * kSensH * kSensH + 4 * (3 * kSensH + 4);

// Float32 master parameters (training): the layout of the gradients too.
struct SensorP {
    float W1[kSensH * kSensK];
    float b1[kSensH];
    float W2[kSensH * kSensH];
    float b2[kSensH];
    float w3[kSensH];
    float b3;
};
constexpr int kSensParams = sizeof(SensorP) / sizeof(float);

// The five features of one quantity from its values at c-2 .. c+2: the shape of the stencil, (v_k - v0) / M for the four
// neighbours with M = max_k |v_k - v0| (0 when the stencil is flat), attenuated by g = min(1, 1e4 M / s) (the shape of a
// variation that is negligible against the quantity's physical scale s > 0, grid-scale noise of amplitude 1e-6 s for
// instance, does not matter and must not look like a jump), and its amplitude log2(1 + 1e4 M / s) / 4. f[2] is the
// amplitude.
__device__ __forceinline__ void sensor_quantity_features(const float v[5], float scale, float f[5]) {
    float M = 0.0f;
    const float v0 = v[2];
#pragma unroll
    for (int k = 0; k < 5; ++k) M = fmaxf(M, fabsf(v[k] - v0));
    const float a = 1e4f * M / scale;
    const float g = fminf(1.0f, a);
    const float iM = M > 0.0f ? g / M : 0.0f;
#pragma unroll
    for (int k = 0; k < 5; ++k) f[k] = (v[k] - v0) * iM;
    f[2] = 0.25f * __log2f(1.0f + a);
}

// The physical scale of sensor quantity sq (rho, u_n, u_t1, u_t2, p) at a cell of density rho and pressure p: rho, the
// sound speed sqrt(gamma (p + p_inf) / rho), p + p_inf (rho and p + p_inf taken at least 1e-30).
template <typename T> __device__ __forceinline__ T sensor_scale(int sq, T rho, T p, T gamma, T p_inf) {
    const T tiny = T(1e-30);
    const T r = rho > tiny ? rho : tiny, pp = p + p_inf > tiny ? p + p_inf : tiny;
    if (sq == 0) return r;
    if (sq == 4) return pp;
    return sqrt(gamma * pp / r);
}

// Index of sensor quantity sq (rho, u_n, u_t1, u_t2, p) among the primitive variables [rho, u, v, p(, w)] for a sweep
// along `axis`; -1 for a velocity the mesh does not have (w on a 2-D mesh).
template <int NV> __device__ __forceinline__ int sensor_var(int sq, int axis) {
    if (sq == 0) return 0;
    if (sq == 4) return 3;
    const int k = (sq - 1 + axis) % 3;   // velocity component: axis 0 (u, v, w), axis 1 (v, w, u), axis 2 (w, u, v)
    return k == 0 ? 1 : (k == 1 ? 2 : (NV == 5 ? 4 : -1));
}

// |WENO5-Z - linear| of the value right of c2 from c0 .. c4 (double precision: the reference's weno5z against the linear
// fifth-order upwind value (2 c0 - 13 c1 + 47 c2 + 27 c3 - 3 c4) / 60).
__device__ __forceinline__ double weno5z_face_gap(double c0, double c1, double c2, double c3, double c4, double eps_rel) {
    const double lin = (2.0 * c0 - 13.0 * c1 + 47.0 * c2 + 27.0 * c3 - 3.0 * c4) / 60.0;
    return fabs(weno5z(c0, c1, c2, c3, c4, eps_rel) - lin);
}

// ------------------------------------------------------------------------------------------------ bf16 helpers
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float round_bf16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

}   // namespace fvg
