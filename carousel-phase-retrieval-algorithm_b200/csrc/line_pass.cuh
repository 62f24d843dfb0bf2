// Helpers shared by the line-pass kernels for planes larger than one CTA
// (kernels_large.cu, kernels_dm_large.cu): asynchronous tile staging, the
// (-1)^n sign flip of the folded fftshift, and an order-preserving float key.
#pragma once
#include "fft_line.cuh"

namespace cpra_b200 {

// Threads per line of the line transforms at 256 and 512 (R = L / 16 values
// per thread).  The per-operator axis passes (kernels_fft.cu) use the same
// split, so line passes built from the same LineFFT steps round identically.
template <int L>
struct LineGeom {
    static constexpr int TPL = 16;
    static constexpr int R = L / TPL;
    static constexpr int J = R / TPL;
    using F = LineFFT<float, L, TPL>;
    __device__ __forceinline__ static int split_pos(int q, int j, int s) { return q + TPL * j + R * s; }
};

__device__ __forceinline__ Cx<float> flip(Cx<float> z, int n) { return (n & 1) ? Cx<float>{-z.x, -z.y} : z; }

// order-preserving map of a float to an unsigned int (maximum by atomicMax)
__device__ __forceinline__ unsigned int ordered(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// asynchronous global -> shared copies (cp.async; completion by wait_group)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// contiguous bytes (a multiple of 16; both addresses 16-byte aligned when
// `vec`, else 4-byte aligned)
__device__ __forceinline__ void stage(void* dst, const void* src, uint32_t bytes, bool vec, int t, int nt) {
    char* d = static_cast<char*>(dst);
    const char* s = static_cast<const char*>(src);
    if (vec)
        for (uint32_t i = 16u * t; i < bytes; i += 16u * nt) cp_async16(d + i, s + i);
    else
        for (uint32_t i = 4u * t; i < bytes; i += 4u * nt) cp_async4(d + i, s + i);
}

}  // namespace cpra_b200
