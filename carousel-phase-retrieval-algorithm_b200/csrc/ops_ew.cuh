// Element-wise operator arithmetic shared by the per-operator kernels and the
// fused difference-map kernel (so both round identically).  Each follows the
// reference operator it names, with T-precision arithmetic and no contraction.
#pragma once
#include "cpra_common.cuh"
#include "cpra_internal.h"

namespace cpra_b200 {

__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float sqrt_rn(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sqrt_rn(double a) { return __dsqrt_rn(a); }

// MKL_Impl.inl:83 zeroes the real part when `S < 0.9` with S promoted to
// double.  For a float S that is exactly `S <= 0.9f` (0.9f < 0.9 <
// nextafter(0.9f, 1)); NaN keeps its value in both forms.
__device__ __forceinline__ bool space_zero(float s) { return s <= 0.9f; }
__device__ __forceinline__ bool space_zero(double s) { return s < 0.9; }

// SpaceConstraint: MKL_Impl.inl:70-84 (threshold) or CUDA_Impl_Kernel.cuh:16-28
// (positivity, real part scaled by the mask value).
template <typename T>
__device__ __forceinline__ Cx<T> space_apply(Cx<T> z, T s, int mode) {
    if (mode == SPACE_THRESHOLD) return {space_zero(s) ? T(0) : z.x, T(0)};
    return {z.x < T(0) ? T(0) : mul_rn(z.x, s), T(0)};
}

__device__ __forceinline__ float rsqrt_fast(float a) { return rsqrtf(a); }
__device__ __forceinline__ double rsqrt_fast(double a) { return rsqrt(a); }

// DataConstraint (real modulus): MKL_Impl.inl:86-106.  A == 0 leaves the value
// unconstrained (DATA_SKIP_ZERO; the CUDA kernel, CUDA_Impl_Kernel.cuh:30-38,
// has no such skip: DATA_ALWAYS); |z|^2 == 0 leaves it unchanged; otherwise
// z <- A * z / |z|, which is std::polar(A, std::arg(z)) up to rounding (the
// reciprocal square root is CUDA's rsqrt, a few ulp like the reference's
// atan2/cos/sin; |z|^2 overflowing to infinity takes the hypot route).
// a / |z| when |z|^2 overflows: out of line, so that the common path stays
// a few instructions in every kernel that inlines data_apply
template <typename T>
__device__ __noinline__ T modulus_ratio_overflow(T a, T x, T y) { return div_rn(a, hypot(x, y)); }

template <typename T>
__device__ __forceinline__ Cx<T> data_apply(Cx<T> z, T a, int mode) {
    if (mode == DATA_SKIP_ZERO && a == T(0)) return z;
    const T n = add_rn(mul_rn(z.x, z.x), mul_rn(z.y, z.y));
    if (!(n > T(0))) return z;
    T r;
    if (isinf(n))
        r = modulus_ratio_overflow(a, z.x, z.y);
    else
        r = mul_rn(a, rsqrt_fast(n));
    return {mul_rn(z.x, r), mul_rn(z.y, r)};
}

// DataConstraint (complex): MKL_Impl.inl:108-126, z <- C where |C|^2 != 0
template <typename T>
__device__ __forceinline__ Cx<T> data_apply_complex(Cx<T> z, Cx<T> c) {
    const T n = add_rn(mul_rn(c.x, c.x), mul_rn(c.y, c.y));
    return (n != T(0)) ? c : z;
}

// MergeAddData: dst <- alpha*src + beta*dst (cblas_?axpby with real
// coefficients, MKL_Impl.inl:31-50), each product and the sum rounded.
template <typename T>
__device__ __forceinline__ Cx<T> merge_apply(Cx<T> src, Cx<T> dst, T alpha, T beta) {
    return {add_rn(mul_rn(alpha, src.x), mul_rn(beta, dst.x)), add_rn(mul_rn(alpha, src.y), mul_rn(beta, dst.y))};
}

}  // namespace cpra_b200
