// One L x L complex plane resident in one CTA's shared memory.
//
// TPL*L threads (TPL = 4, or 8 for the float 128 x 128 plane); thread t works
// on one line (a row in row passes, a column in column passes) as rank
// q = t % TPL of a TPL-thread group inside one warp.  The plane lives in `buf`
// with row stride LS, padding that keeps every pass's accesses of a half-warp
// on distinct banks:
//   TPL = 4: LS = L + 4; a warp's 8 groups take 8 consecutive lines in both
//            passes;
//   TPL = 8: LS = L + 2; a column pass's warp takes 4 consecutive columns,
//            a row pass's warp takes rows r, r + 4, r + 8, r + 12 (the two
//            rows of a half-warp are 4 apart, so their 8 + 8 slots fall on
//            16 distinct bank pairs at this stride).
//
// The per-operator transforms (Forward2D / Backward2D) and the fused
// difference-map kernel are built from the same four steps below, so they
// perform identical arithmetic.  A row thread always sees its row in the
// split layout (elements q + 4j + R s), both as transform input and output,
// so the fused kernel can keep a row's values in registers across passes:
//   forward : rows split->natural (to buf), columns natural->split (registers)
//   inverse : columns split->natural (to buf), rows natural->split (registers)
#pragma once
#include "fft_line.cuh"

namespace cpra_b200 {

template <typename T, int L, int TPL_ = 4>
struct Plane {
    static constexpr int TPL = TPL_;
    static_assert(TPL == 4 || TPL == 8, "4 or 8 threads per line");
    static constexpr int R = L / TPL;
    static constexpr int J = R / TPL;
    static constexpr int LS = (TPL == 8) ? L + 2 : L + TPL;
    static constexpr int NT = L * TPL;
    using F = LineFFT<T, L, TPL>;

    // the line of thread t in row passes and in column passes, and its rank
    __device__ __forceinline__ static int row_of(int t) {
        if constexpr (TPL == 8)
            return ((t >> 7) << 4) + ((t >> 5) & 3) + 4 * ((t >> 3) & 3);
        else
            return t / TPL;
    }
    __device__ __forceinline__ static int col_of(int t) { return t / TPL; }
    __device__ __forceinline__ static int rank_of(int t) { return t % TPL; }

    static constexpr int TW_ENTRIES = F::TW_ENTRIES;

    static constexpr size_t buf_bytes() { return sizeof(Cx<T>) * (size_t)L * LS; }
    static constexpr size_t tw_bytes() { return sizeof(Cx<T>) * (size_t)TW_ENTRIES; }

    // column / row index of output element (j, s) of rank q in split layout
    __device__ __forceinline__ static int split_pos(int q, int j, int s) { return q + TPL * j + R * s; }

    // rows: natural registers of row r -> transformed row, natural, in buf
    template <bool INV>
    __device__ __forceinline__ static void rows_to_buf(Cx<T> (&v)[R], Cx<T>* buf, const Cx<T>* tw, int r, int q) {
        Cx<T> o[J][TPL];
        F::template natural_to_split<INV>(v, o, buf + r * LS, 1, tw, q);
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) buf[r * LS + split_pos(q, j, s)] = o[j][s];
    }

    // rows: split registers of row r -> transformed row, natural, in buf
    template <bool INV>
    __device__ __forceinline__ static void rows_split_to_buf(Cx<T> (&o)[J][TPL], Cx<T>* buf, const Cx<T>* tw, int r,
                                                             int q) {
        Cx<T> v[R];
        F::template split_to_natural<INV>(o, v, buf + r * LS, 1, tw, q);
#pragma unroll
        for (int i = 0; i < R; ++i) buf[r * LS + q + TPL * brev<R>(i)] = v[i];
    }

    // columns: column c natural in buf -> transformed column in split registers
    template <bool INV>
    __device__ __forceinline__ static void col_from_buf(Cx<T> (&o)[J][TPL], Cx<T>* buf, const Cx<T>* tw, int c,
                                                        int q) {
        Cx<T> v[R];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = buf[(q + TPL * k) * LS + c];
        F::template natural_to_split<INV>(v, o, buf + c, LS, tw, q);
    }

    // columns: split registers of column c -> transformed column, natural, in buf
    template <bool INV>
    __device__ __forceinline__ static void col_to_buf(Cx<T> (&o)[J][TPL], Cx<T>* buf, const Cx<T>* tw, int c,
                                                      int q) {
        Cx<T> v[R];
        F::template split_to_natural<INV>(o, v, buf + c, LS, tw, q);
#pragma unroll
        for (int i = 0; i < R; ++i) buf[(q + TPL * brev<R>(i)) * LS + c] = v[i];
    }

    // rows: row r natural in buf -> transformed row in split registers
    template <bool INV>
    __device__ __forceinline__ static void row_from_buf(Cx<T> (&o)[J][TPL], Cx<T>* buf, const Cx<T>* tw, int r,
                                                        int q) {
        Cx<T> v[R];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = buf[r * LS + q + TPL * k];
        F::template natural_to_split<INV>(v, o, buf + r * LS, 1, tw, q);
    }
};

// Threads per line of the single-CTA plane transforms: 8 for the float
// 128 x 128 plane (1024 threads, 16 values each), else 4.  Every kernel that
// transforms such a plane (the per-operator transforms and the fused
// difference map) uses this split, so they round identically.
template <typename T, int L>
__host__ __device__ constexpr int plane_tpl() { return (sizeof(T) == 4 && L == 128) ? 8 : 4; }

// x * (-1)^n, exact
template <typename T>
__device__ __forceinline__ Cx<T> csign(Cx<T> a, int n) { return (n & 1) ? Cx<T>{-a.x, -a.y} : a; }

}  // namespace cpra_b200
