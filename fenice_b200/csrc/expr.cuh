// The evaluator of expr.h's postfix programs, one function for the host and the device: compiled for the host it calls
// the C library's functions (the reference's TinyExpr calls the same ones, so host values carry the reference's bits),
// compiled for the device CUDA's (each within its documented ulp bound of the correctly rounded value).
#pragma once

#include <climits>
#include <cmath>

#include "expr.h"

namespace fvg {
namespace expr {

// TinyExpr's fac, ncr and npr (cpp/third_party/tinyexpr/tinyexpr.c:133-161): integer products in unsigned long
// (64 bits here), infinity when they would overflow, NaN for a negative argument.
__host__ __device__ inline double fac(double a) {
    if (!(a >= 0.0)) return NAN;
    if (a > (double)UINT_MAX) return INFINITY;
    const unsigned int ua = (unsigned int)a;
    unsigned long result = 1;
    for (unsigned long i = 1; i <= ua; ++i) {
        if (i > ULONG_MAX / result) return INFINITY;
        result *= i;
    }
    return (double)result;
}

__host__ __device__ inline double ncr(double n, double r) {
    if (!(n >= 0.0) || !(r >= 0.0) || n < r) return NAN;
    if (n > (double)UINT_MAX || r > (double)UINT_MAX) return INFINITY;
    unsigned long un = (unsigned int)n, ur = (unsigned int)r;
    unsigned long result = 1;
    if (ur > un / 2) ur = un - ur;
    for (unsigned long i = 1; i <= ur; ++i) {
        if (result > ULONG_MAX / (un - ur + i)) return INFINITY;
        result *= un - ur + i;
        result /= i;
    }
    return (double)result;
}

// the logical operators return 1 or 0 as C's int comparisons do; their negated forms -1 or +0
__host__ __device__ inline double apply1(int op, double a) {
    switch (op) {
    case kNeg: return -a;
    case kNot: return (double)(a == 0.0);
    case kNotNot: return (double)(a != 0.0);
    case kNegNot: return (double)(-(int)(a == 0.0));
    case kNegNotNot: return (double)(-(int)(a != 0.0));
    case kAbs: return fabs(a);
    case kAcos: return acos(a);
    case kAsin: return asin(a);
    case kAtan: return atan(a);
    case kCeil: return ceil(a);
    case kCos: return cos(a);
    case kCosh: return cosh(a);
    case kExp: return exp(a);
    case kFac: return fac(a);
    case kFloor: return floor(a);
    case kLn: return log(a);
    case kLog10: return log10(a);
    case kSin: return sin(a);
    case kSinh: return sinh(a);
    case kSqrt: return sqrt(a);
    case kTan: return tan(a);
    case kTanh: return tanh(a);
    default: return NAN;
    }
}

__host__ __device__ inline double apply2(int op, double a, double b) {
    switch (op) {
    case kAdd: return a + b;
    case kSub: return a - b;
    case kMul: return a * b;
    case kDiv: return a / b;
    case kMod: return fmod(a, b);
    case kPow: return pow(a, b);
    case kAtan2: return atan2(a, b);
    case kNcr: return ncr(a, b);
    case kNpr: return ncr(a, b) * fac(b);
    case kGt: return (double)(a > b);
    case kGe: return (double)(a >= b);
    case kLt: return (double)(a < b);
    case kLe: return (double)(a <= b);
    case kEq: return (double)(a == b);
    case kNe: return (double)(a != b);
    case kAnd: return (double)(a != 0.0 && b != 0.0);
    case kOr: return (double)(a != 0.0 || b != 0.0);
    case kComma: return b;
    default: return NAN;
    }
}

// table_value (cpp/src/SimulationInternal.hpp:101-111) of the table at pool[off]: the first or last value outside its
// times, else linear between the rows around t (the first row whose time exceeds t, and the one before). A time that
// is not finite gives NaN (the reference throws).
__host__ __device__ inline double table_value(const double* pool, int off, double t) {
    const int n = (int)pool[off];
    const double* T = pool + off + 1;
    const double* V = T + n;
    if (!isfinite(t)) return NAN;
    if (t <= T[0]) return V[0];
    if (t >= T[n - 1]) return V[n - 1];
    int lo = 0, hi = n - 1;   // T[lo] <= t < T[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (t < T[mid]) hi = mid;
        else lo = mid;
    }
    const double f = (t - T[lo]) / (T[hi] - T[lo]);
    return V[lo] + f * (V[hi] - V[lo]);
}

// Runs the program that starts at code[pc] at (x, y, z, t).
__host__ __device__ inline double run(const Op* code, const double* pool, int pc, double x, double y, double z, double t) {
    double st[kMaxStack];
    int sp = 0;
    for (;; ++pc) {
        const Op o = code[pc];
        if (o.code == kEnd) break;
        if (o.code == kConst) {
            st[sp++] = pool[o.arg];
        } else if (o.code == kVar) {
            st[sp++] = o.arg == kVarX ? x : o.arg == kVarY ? y : o.arg == kVarZ ? z : t;
        } else if (o.code == kTable) {
            st[sp - 1] = table_value(pool, o.arg, st[sp - 1]);
        } else if (o.code >= kAdd) {
            --sp;
            st[sp - 1] = apply2(o.code, st[sp - 1], st[sp]);
        } else {
            st[sp - 1] = apply1(o.code, st[sp - 1]);
        }
    }
    return sp > 0 ? st[sp - 1] : NAN;
}

}  // namespace expr
}  // namespace fvg
