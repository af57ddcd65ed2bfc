// gc_device.cuh — device helpers with the reference's FP64 semantics.
//
// Translation units that include this header are compiled with
// -fmad=false: every `a*b+c` is two roundings, as Julia evaluates it
// without @fastmath.  Where the reference does fuse (scalar @fastmath axpy,
// src/Utils.jl:19-29) the code calls fma() explicitly.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gc_internal.h"

namespace gc {

// Julia `min`/`max` on Float64 (NaN propagates; min(-0.0, 0.0) == -0.0).
__device__ __forceinline__ double jmin(double a, double b) {
    if (isnan(a) || isnan(b)) return a - b;
    if (a < b) return a;
    if (b < a) return b;
    return signbit(a) ? a : b;
}
__device__ __forceinline__ double jmax(double a, double b) {
    if (isnan(a) || isnan(b)) return a - b;
    if (a > b) return a;
    if (b > a) return b;
    return signbit(a) ? b : a;
}

// Julia floor(Int, v); false when v is not representable (InexactError).
__device__ __forceinline__ bool floor_i64(double v, int64_t* out) {
    double f = floor(v);
    if (!(f >= -9.2233720368547758e18 && f < 9.2233720368547758e18)) return false;
    *out = (int64_t)f;
    return true;
}

// Order-preserving map of doubles to uint64 for atomic min/max
// (-0.0 orders below +0.0, matching Julia's min/max on zeros).
__device__ __forceinline__ unsigned long long ord_key(double d) {
    long long b = __double_as_longlong(d);
    return b >= 0 ? ((unsigned long long)b ^ 0x8000000000000000ull) : ~(unsigned long long)b;
}
__device__ __forceinline__ double ord_val(unsigned long long k) {
    long long b = (k & 0x8000000000000000ull) ? (long long)(k ^ 0x8000000000000000ull) : (long long)~k;
    return __longlong_as_double(b);
}

// Compensated x^n for integer n: power by squaring with the rounding error
// of each product carried in a second word (Graillat, Langlois & Louvet,
// 2009).  Same algorithm and operation order as the CPU oracle.
__device__ __forceinline__ double comp_powi(double x, int64_t n) {
    if (n == 0) return 1.0;
    if (n == 3) return x * x * x;
    double xl = 0.0;
    if (n < 0) {
        double rx = 1.0 / x;
        if (n == -2) return rx * rx;
        if (isfinite(x)) xl = -fma(x, rx, -1.0) * rx;
        x = rx;
        n = -n;
    }
    double y = 1.0, yl = 0.0;
    while (n > 1) {
        if (n & 1) {
            double err = y * xl + x * yl;
            double p = x * y;
            double e = fma(x, y, -p);
            y = p;
            yl = e + err;
        }
        double err = x * 2.0 * xl;
        double p = x * x;
        double e = fma(x, x, -p);
        x = p;
        xl = e + err;
        n >>= 1;
    }
    double err = y * xl + x * yl;
    if (isfinite(x) && isfinite(err)) return fma(x, y, err);
    return x * y;
}

// ------------------------------------------------------------ SPH kernels
// src/Kernels.jl:70-81 (cubic spline), :142-153 (Wendland C2; a^4 as (a²)²)
template <int KK>
__device__ __forceinline__ double kernel_w(double norm, double q) {
    if (KK == GC_KERNEL_CUBIC_SPLINE) {
        double a = jmax(0.0, 2.0 - q), b = jmax(0.0, 1.0 - q);
        return norm * (0.25 * (a * a * a) - (b * b * b));
    } else {
        double a = jmax(0.0, 2.0 - q);
        double a2 = a * a;
        return (norm * (a2 * a2)) * (2.0 * q + 1.0);
    }
}
template <int KK>
__device__ __forceinline__ double kernel_dw_dq(double norm, double q) {
    if (KK == GC_KERNEL_CUBIC_SPLINE) {
        double a = jmax(0.0, 2.0 - q), b = jmax(0.0, 1.0 - q);
        return norm * (-3.0 * (0.25 * (a * a) - (b * b)));
    } else {
        double a = jmax(0.0, 2.0 - q);
        return ((-norm * 10.0) * q) * (a * a * a);
    }
}

template <int ND>
__device__ __forceinline__ double dotv(const double* a, const double* b) {
    double s = a[0] * b[0];
#pragma unroll
    for (int d = 1; d < ND; ++d) s = s + a[d] * b[d];
    return s;
}

// src/PairwisePhysics.jl:29-34.  When dot(dx,dv) >= 0 the result is -0.0
// exactly (muv == 0), so the divisions are skipped.
template <int ND>
__device__ __forceinline__ double art_visc(const double* dx, const double* dv, double rr, double h, double ri,
                                           double rj, double alpha, double beta, double ci, double cj) {
    double vr = jmin(dotv<ND>(dx, dv), 0.0);
    if (vr == 0.0 && !signbit(vr) && h > 0.0) {
        // muv = (h*0)/(positive) = +0 exactly; the quotient of a signed zero
        // by a positive finite denominator is that signed zero.
        double mc = 0.5 * (ci + cj);
        double t = (beta * 0.0 - alpha * mc) * 0.0;
        double den = (0.5 * ri) * rj;
        return den > 0.0 ? t : t / den;
    }
    double muv = (h * vr) / (rr + (h * h) * 0.01);
    double mc = 0.5 * (ci + cj);
    return ((beta * muv - alpha * mc) * muv) / ((0.5 * ri) * rj);
}

// src/PairwisePhysics.jl:238-243
template <int ND>
__device__ __forceinline__ double diffusion(const double* dx, double rr, double ri, double rj, double ci,
                                            double cj, double hi, double hj, const double* gx, double delta) {
    double c = 0.5 * (ci + cj);
    double h = 0.5 * (hi + hj);
    return (((((2.0 * delta) * c) * h) * (ri - rj)) * dotv<ND>(dx, gx)) / rr;
}

// src/PairwisePhysics.jl:258-263
template <int ND>
__device__ __forceinline__ double lennard_jones(const double* dx, double rr, double cutoff, double c) {
    double r = sqrt(rr);
    double ind = r < cutoff ? 1.0 : 0.0;
    double f = (ind * (comp_powi(cutoff / r, 12) - comp_powi(cutoff / r, 6))) / rr;
    return ((0.01 * c) * c) * f;
}

}  // namespace gc
