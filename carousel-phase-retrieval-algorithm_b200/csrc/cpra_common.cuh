// Shared device helpers of the B200 carousel phase-retrieval backend:
// the complex value type, separately rounded arithmetic, and launch sizing.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "twiddles_gen.cuh"

namespace cpra_b200 {

// Complex value with the layout of std::complex<T> (interleaved re, im).
template <typename T>
struct alignas(2 * sizeof(T)) Cx {
    T x, y;
};

// Explicitly rounded arithmetic.  The reference evaluates every product and
// sum separately (no fused multiply-add), and the fused kernels must round
// exactly like the per-operator kernels so that both paths agree bit for bit.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

template <typename T>
__device__ __forceinline__ Cx<T> cadd(Cx<T> a, Cx<T> b) { return {add_rn(a.x, b.x), add_rn(a.y, b.y)}; }
template <typename T>
__device__ __forceinline__ Cx<T> csub(Cx<T> a, Cx<T> b) { return {sub_rn(a.x, b.x), sub_rn(a.y, b.y)}; }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// Twiddle products inside the transforms: (a.x + i a.y)(w.x + i w.y) as one
// product and one fused multiply-add per component, written out explicitly so
// that every kernel that transforms a line rounds identically.
template <typename T>
__device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> w) {
    return {fma_rn(a.x, w.x, -mul_rn(a.y, w.y)), fma_rn(a.x, w.y, mul_rn(a.y, w.x))};
}
// a * conj(w)
template <typename T>
__device__ __forceinline__ Cx<T> cmulc(Cx<T> a, Cx<T> w) {
    return {fma_rn(a.x, w.x, mul_rn(a.y, w.y)), fma_rn(a.y, w.x, -mul_rn(a.x, w.y))};
}
template <typename T>
__device__ __forceinline__ Cx<T> cscale(Cx<T> a, T s) { return {mul_rn(a.x, s), mul_rn(a.y, s)}; }
template <typename T>
__device__ __forceinline__ Cx<T> cneg(Cx<T> a) { return {-a.x, -a.y}; }

template <typename T>
__host__ __device__ __forceinline__ constexpr T tw32_cos(int k);
template <typename T>
__host__ __device__ __forceinline__ constexpr T tw32_sin(int k);
template <>
__host__ __device__ __forceinline__ constexpr float tw32_cos<float>(int k) { return tw32_cos_f(k); }
template <>
__host__ __device__ __forceinline__ constexpr float tw32_sin<float>(int k) { return tw32_sin_f(k); }
template <>
__host__ __device__ __forceinline__ constexpr double tw32_cos<double>(int k) { return tw32_cos_d(k); }
template <>
__host__ __device__ __forceinline__ constexpr double tw32_sin<double>(int k) { return tw32_sin_d(k); }

// The block index as a fresh read of %ctaid.x, not folded with earlier reads:
// lets a kernel recompute an address late instead of keeping it in a register
// through a long loop.
__device__ __forceinline__ unsigned cta_index() {
    unsigned v;
    asm volatile("mov.u32 %0, %%ctaid.x;" : "=r"(v));
    return v;
}

// Number of SMs of the current device, cached per device by the host code.
int sm_count();

// Grid size for a grid-stride element-wise kernel: enough CTAs to cover the
// work, capped at a whole number of waves over all SMs.
inline unsigned int ew_grid(uint64_t work_items, unsigned int threads, unsigned int ctas_per_sm = 8) {
    uint64_t need = (work_items + threads - 1) / threads;
    uint64_t cap = (uint64_t)sm_count() * ctas_per_sm;
    if (need < 1) need = 1;
    return (unsigned int)(need < cap ? need : cap);
}

}  // namespace cpra_b200
