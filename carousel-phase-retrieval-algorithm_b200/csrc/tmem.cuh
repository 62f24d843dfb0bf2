// Tensor memory (TMEM) as per-thread on-chip storage for iterates.
//
// An sm_100 SM has 256 KB of tensor memory: 128 lanes x 512 columns of 32-bit
// cells, written and read with tcgen05.st / tcgen05.ld.  Nothing on the phase
// retrieval path is a contraction, so the tensor cores never read it; the
// fused kernels use it as a second register file that lasts a whole launch.
// In the 32x32b access shape, warp w of the CTA reaches lanes
// 32*(w % 4) .. 32*(w % 4) + 31 (lane = its warp quarter + lane id), so the
// warps w, w + 4, w + 8, ... of a CTA share a lane quarter and split its
// columns between them.  Each thread then owns a private strip of columns in
// its own lane.
//
// Every load here waits for its data inside the same asm statement
// (tcgen05.wait::ld), so the compiler never sees a register before it holds
// the loaded value.  Each load first waits for the thread's earlier stores
// (tcgen05.wait::st), so a load always sees what the thread stored before it.
// Stores read their source registers when issued.
#pragma once
#include <cstdint>

#include "cpra_common.cuh"

namespace cpra_b200 {

__device__ __forceinline__ uint32_t smem_addr_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Allocation: one whole warp calls tm_alloc (the same warp later calls
// tm_free); the base address lands in *slot (shared memory).  `cols` is a
// power of two in [32, 512].  The permit to allocate again is given up at
// once: a CTA allocates once per launch.
__device__ __forceinline__ void tm_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr_u32(slot)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_free(uint32_t base, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}
// Ordering of tensor-memory operations across a block barrier.
__device__ __forceinline__ void tm_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tm_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Completion of this thread's stores (before the allocation is given back).
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Address of column `col` in the lane quarter of warp `warp`.
__device__ __forceinline__ uint32_t tm_lane_addr(uint32_t base, int warp, int col) {
    return base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)col;
}

// Four complex floats (8 columns) to tensor memory.
__device__ __forceinline__ void tm_st4(uint32_t a, const Cx<float> (&v)[4]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(a),
        "r"(__float_as_uint(v[0].x)), "r"(__float_as_uint(v[0].y)), "r"(__float_as_uint(v[1].x)),
        "r"(__float_as_uint(v[1].y)), "r"(__float_as_uint(v[2].x)), "r"(__float_as_uint(v[2].y)),
        "r"(__float_as_uint(v[3].x)), "r"(__float_as_uint(v[3].y))
        : "memory");
}

// Four complex floats (8 columns) from tensor memory.
__device__ __forceinline__ void tm_ld4(uint32_t a, Cx<float> (&v)[4]) {
    uint32_t r[8];
    asm volatile(
        "{\n\t"
        "tcgen05.wait::st.sync.aligned;\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n\t"
        "}"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(a)
        : "memory");
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = {__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1])};
}

// Four floats (4 columns) to tensor memory.
__device__ __forceinline__ void tm_st4r(uint32_t a, const float (&v)[4]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(__float_as_uint(v[0])),
                 "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3]))
                 : "memory");
}

// Four complex floats (8 columns at a) and four floats (4 columns at b) from
// tensor memory, one wait for both.
__device__ __forceinline__ void tm_ld4_4r(uint32_t a, uint32_t b, Cx<float> (&u)[4], float (&v)[4]) {
    uint32_t r[12];
    asm volatile(
        "{\n\t"
        "tcgen05.wait::st.sync.aligned;\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%12];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%8, %9, %10, %11}, [%13];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n\t"
        "}"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
        : "r"(a), "r"(b)
        : "memory");
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        u[i] = {__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1])};
        v[i] = __uint_as_float(r[8 + i]);
    }
}

}  // namespace cpra_b200
