// One L x L complex plane resident in one CTA's shared memory.
//
// 4*L threads; thread t works on line t/4 (a row in row passes, a column in
// column passes) as rank q = t%4 of a 4-thread group inside one warp.  The
// plane lives in `buf` with row stride LS = L + 4 (padding that keeps the
// natural-order row and column accesses of a half-warp on distinct banks).
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

template <typename T, int L>
struct Plane {
    static constexpr int TPL = 4;
    static constexpr int R = L / TPL;
    static constexpr int J = R / TPL;
    static constexpr int LS = L + TPL;
    static constexpr int NT = L * TPL;
    using F = LineFFT<T, L, TPL>;

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

// x * (-1)^n, exact
template <typename T>
__device__ __forceinline__ Cx<T> csign(Cx<T> a, int n) { return (n & 1) ? Cx<T>{-a.x, -a.y} : a; }

}  // namespace cpra_b200
