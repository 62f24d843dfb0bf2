// Helpers shared by the line-pass kernels for planes larger than one CTA
// (kernels_large.cu, kernels_dm_large.cu): asynchronous tile staging, the
// (-1)^n sign flip of the folded fftshift, and an order-preserving float key.
#pragma once
#include "fft_line.cuh"

namespace cpra_b200 {

// Geometry of the line passes at 256 and 512.  A line is TPL threads of one
// warp with R = 16 values each: 16 threads at 256, 32 at 512 (LineFFT's HALF
// form), so a thread holds 16 complex values at both sizes.  The per-operator
// axis passes (kernels_fft.cu) use the same split, so line passes built from
// the same LineFFT steps round identically.  Outputs of a transform are in the
// flat layout LineFFT::pos.
//   rows:    ROW_LINES lines per 256-thread CTA, each line's L slots of a tile
//            in shared memory (row-major, pitch L).
//   columns: COL_LINES columns per 256-thread CTA in a [L][CS] tile.  At 256
//            two columns share a warp, interleaved lane by lane (line =
//            2 (t >> 5) + (t & 1)), and CS = 18 (16-byte rows): a half-warp's
//            8-byte accesses touch 8 ranks of both columns on 16 distinct bank
//            pairs.  At 512 a warp is one column and CS = 9 (odd, 8-byte rows
//            and copies): a half-warp's 16 consecutive ranks or slots land on
//            16 distinct bank pairs.  The A tile's pitch AS is 20 (16-byte
//            rows) at 256 and 9 at 512 (4-byte copies; odd, so a warp's 32
//            rows of one column hit 32 distinct banks).
template <int L>
struct LineGeom {
    static constexpr int TPL = (L >= 512) ? 32 : 16;
    static constexpr int R = L / TPL;
    using F = LineFFT<float, L, TPL>;
    static constexpr int THREADS = 256;
    static constexpr int ROW_LINES = THREADS / TPL;
    static constexpr int COL_LINES = THREADS / TPL;
    static constexpr bool PAIRED = (TPL == 16);  // two columns per warp
    static constexpr int CS = PAIRED ? COL_LINES + 2 : COL_LINES + 1;
    static constexpr int AS = PAIRED ? COL_LINES + 4 : COL_LINES + 1;
    static constexpr size_t row_tile = (size_t)ROW_LINES * L;  // elements
    static_assert(R == 16, "16 values per thread");
    static_assert(L % ROW_LINES == 0 && L % COL_LINES == 0, "a CTA's lines must belong to one pattern");
    __device__ __forceinline__ static int pos(int q, int i) { return F::pos(q, i); }
    // (line, rank) of thread t in a row pass and in a column pass
    __device__ __forceinline__ static void row_lane(int t, int& line, int& q) {
        line = t / TPL;
        q = t % TPL;
    }
    __device__ __forceinline__ static void col_lane(int t, int& line, int& q) {
        if constexpr (PAIRED) {
            line = 2 * (t >> 5) + (t & 1);
            q = (t & 31) >> 1;
        } else {
            line = t >> 5;
            q = t & 31;
        }
    }
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
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
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

// First tile row of the thread with copy-row index r when a pass of the CTA
// copies `step` rows.  With 32 rows per pass and 8 copies per row (512: odd
// pitch 9, 8-byte complex and 4-byte A copies) a warp takes rows w, w + 8,
// w + 16, w + 24 of each 32-row block: at pitch 9 their slots fall on
// distinct bank pairs per half-warp (complex) and distinct banks (A), where
// four consecutive rows would put two copies on one bank.  Any other step
// keeps consecutive rows.  A bijection on 0..step-1 either way.
__device__ __forceinline__ int tile_row(int r, int step) { return step == 32 ? (r >> 2) + 8 * (r & 3) : r; }

// A column tile: rows n < L of LN consecutive complex at src + n * ld into
// dst + n * CS (16-byte copies when CS is even, 8-byte copies otherwise), and
// optionally LN floats per row of A at a + n * ld into as + n * AS (16-byte
// copies when `avec` and AS % 4 == 0, else 4-byte copies).  `nt` (the CTA's
// threads) is a multiple of the chunks per row, so every thread keeps one
// chunk position k of a row and walks the rows n = t / chunks + (nt / chunks) j
// by pointer steps.
template <int L, int LN, int CS, int AS>
__device__ __forceinline__ void stage_col_tile(Cx<float>* dst, const Cx<float>* src, float* as, const float* a,
                                               uint64_t ld, bool avec, int t, int nt) {
    constexpr int W = (CS % 2 == 0) ? 2 : 1;  // complex per copy
    constexpr int CH = LN / W;
    {
        const int k = t % CH, step = nt / CH, n0 = (W == 1) ? tile_row(t / CH, step) : t / CH;
        const Cx<float>* s = src + (uint64_t)n0 * ld + W * k;
        Cx<float>* d = dst + n0 * CS + W * k;
        const uint64_t sstep = (uint64_t)step * ld;
        for (int n = n0; n < L; n += step, s += sstep, d += step * CS) {
            if constexpr (W == 2)
                cp_async16(d, s);
            else
                cp_async8(d, s);
        }
    }
    if (!a) return;
    if (AS % 4 == 0 && avec) {
        constexpr int CA = LN / 4;
        const int k = t % CA, n0 = t / CA, step = nt / CA;
        const float* s = a + (uint64_t)n0 * ld + 4 * k;
        float* d = as + n0 * AS + 4 * k;
        const uint64_t sstep = (uint64_t)step * ld;
        for (int n = n0; n < L; n += step, s += sstep, d += step * AS) cp_async16(d, s);
    } else {
        const int k = t % LN, step = nt / LN, n0 = tile_row(t / LN, step);
        const float* s = a + (uint64_t)n0 * ld + k;
        float* d = as + n0 * AS + k;
        const uint64_t sstep = (uint64_t)step * ld;
        for (int n = n0; n < L; n += step, s += sstep, d += step * AS) cp_async4(d, s);
    }
}

// the tile back: rows of LN complex from src + n * CS to dst + n * ld, by the
// same per-thread walk
template <int L, int LN, int CS>
__device__ __forceinline__ void store_col_tile(Cx<float>* dst, const Cx<float>* src, uint64_t ld, int t, int nt) {
    constexpr int W = (CS % 2 == 0) ? 2 : 1;
    constexpr int CH = LN / W;
    const int k = t % CH, step = nt / CH, n0 = (W == 1) ? tile_row(t / CH, step) : t / CH;
    Cx<float>* d = dst + (uint64_t)n0 * ld + W * k;
    const Cx<float>* s = src + n0 * CS + W * k;
    const uint64_t dstep = (uint64_t)step * ld;
    for (int n = n0; n < L; n += step, d += dstep, s += step * CS) {
        if constexpr (W == 2)
            *reinterpret_cast<float4*>(d) = *reinterpret_cast<const float4*>(s);
        else
            *d = *s;
    }
}

}  // namespace cpra_b200
