// Device physics of the finite-volume path: equation of state, TVD limiters, WENO-Z reconstruction and the
// HLLC-family Riemann solvers, written for sm_100a.
//
// Every function keeps the operation order of the reference (Fenice, cpp/include/fv/Core.hpp,
// cpp/include/fv/Schemes.hpp, cpp/src/Schemes.cpp) and the library is compiled with --fmad=false, so the FP64
// instantiation gives the reference's bits: IEEE-rounded add, mul, div and sqrt, no contraction into fused
// multiply-adds. std::max / std::min are the ternaries `a < b ? b : a` / `b < a ? b : a` (fmax would pick the
// other operand for NaN and signed zeros).
//
// The functions are templates over the arithmetic type T (double: the plain form; float: the mixed form) and
// over the dimension: a planar (2-D) state has no z-momentum, and every term the reference adds for it is
// exactly +0 there, so dropping it gives the same bits.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace fvg {

constexpr int kFirstOrder = 0, kMuscl = 1, kWeno3 = 2, kWeno5 = 3;
constexpr int kMinmod = 0, kVanLeer = 1, kMC = 2, kKoren = 3;
constexpr int kHLLC = 0, kLowMach = 1;
constexpr int kIdeal = 0, kStiffened = 1;

template <typename T> struct Num;
template <> struct Num<double> {
    static constexpr double eos_eps = 1e-10;   // Core.hpp:169
    static constexpr double denom_eps = 1e-14; // Schemes.cpp:64
    static constexpr double mach_eps = 1e-12;  // Schemes.cpp:66
    static constexpr double weno_floor = 1e-300;
};
template <> struct Num<float> {
    static constexpr float eos_eps = 1e-10f;
    static constexpr float denom_eps = 1e-14f;
    static constexpr float mach_eps = 1e-12f;
    static constexpr float weno_floor = 1e-30f;  // 1e-300 is below the float range
};

template <typename T> __host__ __device__ __forceinline__ T vmax(T a, T b) { return (a < b) ? b : a; }
template <typename T> __host__ __device__ __forceinline__ T vmin(T a, T b) { return (b < a) ? b : a; }

// The equation of state (Core.hpp:173-238): ideal gas p = (gamma-1) rho e, stiffened gas p + gamma p_inf = (gamma-1) rho e.
template <typename T> struct Eos {
    int type;
    T gamma, p_inf;
};

// State of NV components: [rho, rho u, rho v, rho E (, rho w)] or primitive [rho, u, v, p (, w)].
template <typename T, int NV> struct St {
    T v[NV];
    __device__ __forceinline__ T& operator[](int q) { return v[q]; }
    __device__ __forceinline__ const T& operator[](int q) const { return v[q]; }
};

template <typename T> __device__ __forceinline__ T internal_energy(const Eos<T>& e, T p) {
    return e.type == kIdeal ? p / (e.gamma - T(1)) : (p + e.gamma * e.p_inf) / (e.gamma - T(1));
}
template <typename T> __device__ __forceinline__ T pressure(const Eos<T>& e, T rho_e) {
    return e.type == kIdeal ? (e.gamma - T(1)) * rho_e : (e.gamma - T(1)) * rho_e - e.gamma * e.p_inf;
}

// prim_to_cons (Core.hpp:209-215)
template <typename T, int NV> __device__ __forceinline__ St<T, NV> p2c(const Eos<T>& e, const St<T, NV>& W) {
    St<T, NV> U;
    const T rho = W[0], u = W[1], v = W[2], p = W[3];
    T ke;
    if constexpr (NV == 5) {
        const T w = W[4];
        ke = T(0.5) * rho * (u * u + v * v + w * w);
        U[4] = rho * w;
    } else {
        ke = T(0.5) * rho * (u * u + v * v);
    }
    const T en = internal_energy(e, p);
    U[0] = rho;
    U[1] = rho * u;
    U[2] = rho * v;
    U[3] = en + ke;
    return U;
}

// cons_to_prim (Core.hpp:218-227); inv receives 1 / rho of the floored density
template <typename T, int NV> __device__ __forceinline__ St<T, NV> c2p(const Eos<T>& e, const St<T, NV>& U, T& inv) {
    St<T, NV> W;
    const T rho = vmax(U[0], Num<T>::eos_eps);
    inv = T(1) / rho;
    const T u = U[1] * inv, v = U[2] * inv;
    T e_kin;
    if constexpr (NV == 5) {
        const T w = U[4] * inv;
        e_kin = T(0.5) * rho * (u * u + v * v + w * w);
        W[4] = w;
    } else {
        e_kin = T(0.5) * rho * (u * u + v * v);
    }
    const T p = pressure(e, U[3] - e_kin);
    W[0] = rho;
    W[1] = u;
    W[2] = v;
    W[3] = vmax(p, Num<T>::eos_eps);
    return W;
}
template <typename T, int NV> __device__ __forceinline__ St<T, NV> c2p(const Eos<T>& e, const St<T, NV>& U) {
    T inv;
    return c2p(e, U, inv);
}

// sound_speed_inv (Core.hpp:234-237)
template <typename T> __device__ __forceinline__ T sound_speed_inv(const Eos<T>& e, T p, T inv_rho) {
    if (e.type == kIdeal) return sqrt(e.gamma * vmax(p, Num<T>::eos_eps) * inv_rho);
    return sqrt(e.gamma * (p + e.p_inf) * inv_rho);
}
// sound_speed (Core.hpp:229-232)
template <typename T> __device__ __forceinline__ T sound_speed(const Eos<T>& e, T p, T rho) {
    if (e.type == kIdeal) return sqrt(e.gamma * vmax(p, Num<T>::eos_eps) / vmax(rho, Num<T>::eos_eps));
    return sqrt(e.gamma * (p + e.p_inf) / vmax(rho, Num<T>::eos_eps));
}

template <typename T, int NV> __device__ __forceinline__ St<T, NV> round_trip(const Eos<T>& e, const St<T, NV>& U) {
    return p2c(e, c2p(e, U));
}

// ------------------------------------------------------------------ limiters (Schemes.hpp:93-117)
template <typename T> __device__ __forceinline__ T sgn(T x) { return (x > T(0)) ? T(1) : ((x < T(0)) ? T(-1) : T(0)); }
template <typename T> __device__ __forceinline__ T limiter(int l, T a, T b) {
    switch (l) {
    case kMinmod: return T(0.5) * (sgn(a) + sgn(b)) * vmin(fabs(a), fabs(b));
    case kVanLeer: {
        const T ab = a * b;
        return (ab > T(0)) ? T(2) * ab / (a + b) : T(0);
    }
    case kMC:
        if (!(a * b > T(0))) return T(0);
        return vmin(vmin(T(2) * fabs(a), T(0.5) * fabs(a + b)), T(2) * fabs(b)) * sgn(a);
    default:
        if (!(a * b > T(0))) return T(0);
        return fmin(fmin(T(2) * fabs(a), fabs(T(2) * a + b) / T(3)), T(2) * fabs(b)) * sgn(a);
    }
}

// ------------------------------------------------------------------ WENO-Z (Borges et al. 2008; Schemes.cpp:328-353)
// The value at the face on the right of c1 from (c0, c1, c2); eps relative to the mean square of the stencil.
template <typename T> __device__ __forceinline__ T weno3z(T c0, T c1, T c2, T eps_rel) {
    const T eps = eps_rel * (c0 * c0 + c1 * c1 + c2 * c2) * (T(1) / T(3)) + Num<T>::weno_floor;
    const T v0 = T(-0.5) * c0 + T(1.5) * c1, v1 = T(0.5) * c1 + T(0.5) * c2;
    const T b0 = (c1 - c0) * (c1 - c0), b1 = (c2 - c1) * (c2 - c1);
    const T tau = fabs(b0 - b1);
    const T a0 = (T(1) / T(3)) * (T(1) + tau / (b0 + eps)), a1 = (T(2) / T(3)) * (T(1) + tau / (b1 + eps));
    return (a0 * v0 + a1 * v1) / (a0 + a1);
}
// The value at the face on the right of c2 from (c0 .. c4).
template <typename T> __device__ __forceinline__ T weno5z(T c0, T c1, T c2, T c3, T c4, T eps_rel) {
    const T eps = eps_rel * (c0 * c0 + c1 * c1 + c2 * c2 + c3 * c3 + c4 * c4) * T(0.2) + Num<T>::weno_floor;
    const T p0 = (T(2) * c0 - T(7) * c1 + T(11) * c2) / T(6);
    const T p1 = (-c1 + T(5) * c2 + T(2) * c3) / T(6);
    const T p2 = (T(2) * c2 + T(5) * c3 - c4) / T(6);
    const T s0 = c0 - T(2) * c1 + c2, t0 = c0 - T(4) * c1 + T(3) * c2;
    const T s1 = c1 - T(2) * c2 + c3, t1 = c1 - c3;
    const T s2 = c2 - T(2) * c3 + c4, t2 = T(3) * c2 - T(4) * c3 + c4;
    const T b0 = (T(13) / T(12)) * s0 * s0 + T(0.25) * t0 * t0;
    const T b1 = (T(13) / T(12)) * s1 * s1 + T(0.25) * t1 * t1;
    const T b2 = (T(13) / T(12)) * s2 * s2 + T(0.25) * t2 * t2;
    const T tau = fabs(b0 - b2);
    const T a0 = T(0.1) * (T(1) + tau / (b0 + eps)), a1 = T(0.6) * (T(1) + tau / (b1 + eps)), a2 = T(0.3) * (T(1) + tau / (b2 + eps));
    return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}
// The single-precision WENO5-Z of the mixed form: the same weights, with every product and sum rounded by an explicit
// intrinsic (FMAs placed by hand) and the candidates' common 1/6 folded into the last division, so that no compiler pass
// contracts it one way in one kernel and another way in the next: every kernel that solves a face gets the same bits.
__device__ __forceinline__ float weno5z(float c0, float c1, float c2, float c3, float c4, float eps_rel) {
    float ss = __fmul_rn(c0, c0);
    ss = __fmaf_rn(c1, c1, ss);
    ss = __fmaf_rn(c2, c2, ss);
    ss = __fmaf_rn(c3, c3, ss);
    ss = __fmaf_rn(c4, c4, ss);
    const float eps = __fmaf_rn(__fmul_rn(eps_rel, ss), 0.2f, Num<float>::weno_floor);
    const float p0 = __fmaf_rn(11.0f, c2, __fmaf_rn(-7.0f, c1, __fmul_rn(2.0f, c0)));   // 6 x the three candidates
    const float p1 = __fmaf_rn(2.0f, c3, __fmaf_rn(5.0f, c2, -c1));
    const float p2 = __fmaf_rn(5.0f, c3, __fmaf_rn(2.0f, c2, -c4));
    const float s0 = __fadd_rn(__fmaf_rn(-2.0f, c1, c0), c2), t0 = __fmaf_rn(3.0f, c2, __fmaf_rn(-4.0f, c1, c0));
    const float s1 = __fadd_rn(__fmaf_rn(-2.0f, c2, c1), c3), t1 = __fsub_rn(c1, c3);
    const float s2 = __fadd_rn(__fmaf_rn(-2.0f, c3, c2), c4), t2 = __fadd_rn(__fmaf_rn(-4.0f, c3, __fmul_rn(3.0f, c2)), c4);
    constexpr float k = 13.0f / 12.0f;
    const float b0 = __fmaf_rn(__fmul_rn(k, s0), s0, __fmul_rn(__fmul_rn(0.25f, t0), t0));
    const float b1 = __fmaf_rn(__fmul_rn(k, s1), s1, __fmul_rn(__fmul_rn(0.25f, t1), t1));
    const float b2 = __fmaf_rn(__fmul_rn(k, s2), s2, __fmul_rn(__fmul_rn(0.25f, t2), t2));
    const float tau = fabsf(__fsub_rn(b0, b2));
    const float a0 = __fmul_rn(0.1f, __fadd_rn(1.0f, tau / __fadd_rn(b0, eps)));
    const float a1 = __fmul_rn(0.6f, __fadd_rn(1.0f, tau / __fadd_rn(b1, eps)));
    const float a2 = __fmul_rn(0.3f, __fadd_rn(1.0f, tau / __fadd_rn(b2, eps)));
    const float num = __fmaf_rn(a2, p2, __fmaf_rn(a1, p1, __fmul_rn(a0, p0)));
    return num / __fmul_rn(6.0f, __fadd_rn(__fadd_rn(a0, a1), a2));
}

// ------------------------------------------------------------------ HLLC (Toro) with Einfeldt bounds (Schemes.cpp:116-200)
template <typename T> __device__ __forceinline__ T safe_denom(T x) { return copysign(vmax(fabs(x), Num<T>::denom_eps), x); }

// The flux along `axis` (0, 1, 2) from the primitive (floored) and conservative states of both sides; returns max(|S_L|, |S_R|).
template <typename T, int NV>
__device__ __forceinline__ T hllc_core(const St<T, NV>& WL, const St<T, NV>& WR, const St<T, NV>& UL, const St<T, NV>& UR, T inv_L,
                                       T inv_R, T c_L, T c_R, int axis, T shock_blend, St<T, NV>& F) {
    constexpr int NA = NV == 5 ? 3 : 2;   // velocity components
    const T rho_L = WL[0], p_L = WL[3];
    const T rho_R = WR[0], p_R = WR[3];
    T vel_L[NA], vel_R[NA];
    vel_L[0] = WL[1];
    vel_L[1] = WL[2];
    vel_R[0] = WR[1];
    vel_R[1] = WR[2];
    if constexpr (NA == 3) {
        vel_L[2] = WL[4];
        vel_R[2] = WR[4];
    }
    const T E_L = UL[3] * inv_L, E_R = UR[3] * inv_R;
    const T Vn_L = vel_L[axis], Vn_R = vel_R[axis];
    const int mn = axis == 0 ? 1 : (axis == 1 ? 2 : 4);
    St<T, NV> FL, FR;
    FL[0] = rho_L * Vn_L;
    FR[0] = rho_R * Vn_R;
#pragma unroll
    for (int a = 0; a < NA; ++a) {
        const int m = a == 0 ? 1 : (a == 1 ? 2 : 4);
        FL[m] = rho_L * vel_L[a] * Vn_L;
        FR[m] = rho_R * vel_R[a] * Vn_R;
    }
    FL[mn] = FL[mn] + p_L;
    FR[mn] = FR[mn] + p_R;
    FL[3] = Vn_L * (rho_L * E_L + p_L);
    FR[3] = Vn_R * (rho_R * E_R + p_R);
    const T S_L = vmin(Vn_L - c_L, Vn_R - c_R);
    const T S_R = vmax(Vn_L + c_L, Vn_R + c_R);
    const T num = rho_R * Vn_R * (S_R - Vn_R) - rho_L * Vn_L * (S_L - Vn_L) + p_L - p_R;
    const T den = rho_R * (S_R - Vn_R) - rho_L * (S_L - Vn_L);
    const T S_M = num / safe_denom(den);
    const T den_star_L = safe_denom(S_L - S_M);
    const T den_star_R = safe_denom(S_R - S_M);
    const T den_pL = safe_denom(S_L - Vn_L);
    const T den_pR = safe_denom(S_R - Vn_R);
    const T fL = rho_L * (S_L - Vn_L) / den_star_L;
    const T fR = rho_R * (S_R - Vn_R) / den_star_R;
    St<T, NV> UsL, UsR;
    UsL[0] = fL;
    UsR[0] = fR;
#pragma unroll
    for (int a = 0; a < NA; ++a) {
        const int m = a == 0 ? 1 : (a == 1 ? 2 : 4);
        UsL[m] = fL * (a == axis ? S_M : vel_L[a]);
        UsR[m] = fR * (a == axis ? S_M : vel_R[a]);
    }
    UsL[3] = fL * (E_L + (S_M - Vn_L) * (S_M + p_L / (rho_L * den_pL)));
    UsR[3] = fR * (E_R + (S_M - Vn_R) * (S_M + p_R / (rho_R * den_pR)));
    // flux selection by wave ordering: the four tests in the reference's sequence (a NaN speed leaves F = 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        T f = T(0);
        if (S_L >= T(0)) f = FL[q];
        if (S_L < T(0) && S_M >= T(0)) f = FL[q] + S_L * (UsL[q] - UL[q]);
        if (S_M < T(0) && S_R >= T(0)) f = FR[q] + S_R * (UsR[q] - UR[q]);
        if (S_R < T(0)) f = FR[q];
        F[q] = f;
    }
    if (shock_blend > T(0)) {
        const T s = fabs(p_R - p_L) / vmin(p_L, p_R);
        if (s > shock_blend) {
            const T phi = vmin((s - shock_blend) / shock_blend, T(1));
            if (S_L >= T(0)) {
#pragma unroll
                for (int q = 0; q < NV; ++q) F[q] = (T(1) - phi) * F[q] + phi * FL[q];
            } else if (S_R <= T(0)) {
#pragma unroll
                for (int q = 0; q < NV; ++q) F[q] = (T(1) - phi) * F[q] + phi * FR[q];
            } else {
                const T inv = T(1) / (S_R - S_L);
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    const T fh = (S_R * FL[q] - S_L * FR[q] + S_L * S_R * (UR[q] - UL[q])) * inv;
                    F[q] = (T(1) - phi) * F[q] + phi * fh;
                }
            }
        }
    }
    return vmax(fabs(S_L), fabs(S_R));
}

// RiemannSolver::face_flux (Schemes.cpp:202-229): HLLC, or Thornber's low-Mach velocity-jump scaling then HLLC.
template <int RIEMANN, typename T, int NV>
__device__ __forceinline__ T face_flux(const Eos<T>& e, T shock_blend, const St<T, NV>& UL, const St<T, NV>& UR, int axis, St<T, NV>& F) {
    T inv_L, inv_R;
    St<T, NV> WL = c2p(e, UL, inv_L);
    St<T, NV> WR = c2p(e, UR, inv_R);
    const T c_L = sound_speed_inv(e, WL[3], inv_L);
    const T c_R = sound_speed_inv(e, WR[3], inv_R);
    if constexpr (RIEMANN == kHLLC) {
        return hllc_core(WL, WR, UL, UR, inv_L, inv_R, c_L, c_R, axis, shock_blend, F);
    } else {
        T mL2 = WL[1] * WL[1] + WL[2] * WL[2], mR2 = WR[1] * WR[1] + WR[2] * WR[2];
        if constexpr (NV == 5) {
            mL2 = mL2 + WL[4] * WL[4];
            mR2 = mR2 + WR[4] * WR[4];
        }
        const T M_L = sqrt(mL2) / (c_L + Num<T>::mach_eps);
        const T M_R = sqrt(mR2) / (c_R + Num<T>::mach_eps);
        const T z = vmin(vmax(vmax(M_L, M_R), T(1e-4)), T(1));
#pragma unroll
        for (int a = 0; a < (NV == 5 ? 3 : 2); ++a) {
            const int m = a == 0 ? 1 : (a == 1 ? 2 : 4);
            const T avg = T(0.5) * (WL[m] + WR[m]);
            const T half = T(0.5) * (WL[m] - WR[m]);
            WL[m] = avg + z * half;
            WR[m] = avg - z * half;
        }
        return hllc_core(WL, WR, p2c(e, WL), p2c(e, WR), inv_L, inv_R, c_L, c_R, axis, shock_blend, F);
    }
}

}   // namespace fvg
