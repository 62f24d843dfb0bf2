// Shifted 2D / 3D transforms (Forward2D, Backward2D, Forward3D, Backward3D).
//
// The reference computes fftshift -> DFT -> fftshift with three passes over
// memory (include/detail/MKL_Impl.inl:128-178, include/detail/CUDA_Impl.inl:
// 20-84).  For even sizes shift o DFT o shift equals s * D (.) DFT(D (.) x)
// with D = (-1)^(sum of indices) and s = (-1)^(sum of half sizes), so here the
// shifts are sign flips applied while the data is in registers:
//   * square planes up to 128 x 128 (float) / 64 x 64 (double): one CTA per
//     plane holds the whole plane in shared memory, one HBM round trip;
//   * other power-of-two lengths up to 1024: one pass per axis, each pass
//     staging a tile of lines in shared memory;
//   * other even lengths: a direct O(L^2) DFT pass per axis.
#include "cpra_internal.h"
#include "fft2d_cta.cuh"
#include "line_pass.cuh"
#include "ops_ew.cuh"

namespace cpra_b200 {

namespace {

// ---------------------------------------------------------------------------
// one plane per CTA
// ---------------------------------------------------------------------------
template <typename T, int L, bool INV>
__global__ void __launch_bounds__(plane_tpl<T, L>() * L) k_plane_fft(Cx<T>* __restrict__ data,
                                                                     const Cx<T>* __restrict__ twg, T scale,
                                                                     int s_neg) {
    using P = Plane<T, L, plane_tpl<T, L>()>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T>* buf = reinterpret_cast<Cx<T>*>(smem_raw);
    Cx<T>* tw = buf + L * P::LS;
    const int t = threadIdx.x, row = P::row_of(t), col = P::col_of(t), q = P::rank_of(t);
    P::F::fill_twiddles(tw, twg, t, P::NT);
    Cx<T>* g = data + (size_t)blockIdx.x * L * L;
    __syncthreads();
    if constexpr (!INV) {
        Cx<T> o[P::J][P::TPL];
#pragma unroll
        for (int j = 0; j < P::J; ++j)
#pragma unroll
            for (int s = 0; s < P::TPL; ++s) {
                const int n = P::split_pos(q, j, s);
                o[j][s] = csign(g[row * L + n], row + n);
            }
        P::template rows_split_to_buf<false>(o, buf, tw, row, q);
        __syncthreads();
        P::template col_from_buf<false>(o, buf, tw, col, q);
#pragma unroll
        for (int j = 0; j < P::J; ++j)
#pragma unroll
            for (int s = 0; s < P::TPL; ++s) {
                const int f = P::split_pos(q, j, s);
                g[f * L + col] = csign(o[j][s], f + col + s_neg);
            }
    } else {
        Cx<T> o[P::J][P::TPL];
#pragma unroll
        for (int j = 0; j < P::J; ++j)
#pragma unroll
            for (int s = 0; s < P::TPL; ++s) {
                const int f = P::split_pos(q, j, s);
                o[j][s] = csign(g[f * L + col], f + col + s_neg);
            }
        P::template col_to_buf<true>(o, buf, tw, col, q);
        __syncthreads();
        P::template row_from_buf<true>(o, buf, tw, row, q);
#pragma unroll
        for (int j = 0; j < P::J; ++j)
#pragma unroll
            for (int s = 0; s < P::TPL; ++s) {
                const int f = P::split_pos(q, j, s);
                g[row * L + f] = csign(cscale(o[j][s], scale), row + f);
            }
    }
}

template <typename T, int L>
cudaError_t plane_fft(void* x, uint64_t batch, bool inverse, T scale, int s_neg, const void* tw, cudaStream_t st) {
    using P = Plane<T, L, plane_tpl<T, L>()>;
    const size_t smem = P::buf_bytes() + P::tw_bytes();
    auto kf = inverse ? k_plane_fft<T, L, true> : k_plane_fft<T, L, false>;
    cudaError_t e = cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kf<<<(unsigned)batch, P::NT, smem, st>>>((Cx<T>*)x, (const Cx<T>*)tw, scale, s_neg);
    count_launches();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// one axis of a [Bo][L][Bi] array, power-of-two L <= 1024
// ---------------------------------------------------------------------------
constexpr int AXIS_THREADS = 256;

// Optional per-line work of an axis pass (the fused 3D constraint step):
//   AXIS_DC_ROUNDTRIP: forward transform, complex DataConstraint with C at
//     each element, inverse transform, with the per-call passes' sign flips in
//     the same order (output flip, constraint, input flip of the inverse);
//   AXIS_SPACE: SpaceConstraint with S on the pass's output.
// aux is indexed as the operators index their constraint, i % aux_plane.
//   AXIS_DCR_ROUNDTRIP: the same with the real modulus DataConstraint (A, data_mode);
//   AXIS_T2_PROLOGUE: the pass's input is t2' = a2*x + b2*SpaceConstraint(t2)
//     (data holds t2; x = x_in, S = aux), the difference map's second half;
//   AXIS_T1_EPILOGUE: the output w becomes SpaceConstraint(a1*x + b1*w) (x = x_in);
//   AXIS_X_EPILOGUE: the output w is t2; x <- a4*w + b4*(a3*t1 + b3*x) (t1 = t1_in).
enum AxisOpKind : int {
    AXIS_PLAIN = 0,
    AXIS_DC_ROUNDTRIP = 1,
    AXIS_SPACE = 2,
    AXIS_DCR_ROUNDTRIP = 3,
    AXIS_T2_PROLOGUE = 4,
    AXIS_T1_EPILOGUE = 5,
    AXIS_X_EPILOGUE = 6
};
struct AxisOp {
    int kind = AXIS_PLAIN;
    const void* aux = nullptr;  // C, A or S
    uint64_t aux_plane = 1;
    int space_mode = 0, data_mode = 0;
    void* x_in = nullptr;       // x of the difference map
    const void* t1_in = nullptr;
    double a = 0.0, b = 0.0, a2 = 0.0, b2 = 0.0;  // merge coefficients (rounded to T by the caller)
};

// Shared tile of an axis pass: AXIS_THREADS / TPL lines of L elements.
// Contiguous axes keep lines as rows of pitch LSX (TPL < 16: padded by TPL so
// the lines of a half-warp fall on distinct bank pairs); strided axes keep
// them as columns of pitch CSX (odd, or 4 mod 16 at TPL = 4), which keeps the
// staging copies, the natural-order loads, the exchange and the outputs on
// distinct bank pairs at every length but 512 and 1024 (2-way there).
template <int L, int TPL>
struct AxisTile {
    static constexpr int LINES = AXIS_THREADS / TPL;
    static constexpr int LSX = L + (TPL < 16 ? TPL : 0);
    static constexpr int CSX = (TPL == 4) ? LINES + 4 : LINES + 1;
    static constexpr int ELEMS = (LINES * LSX > L * CSX) ? LINES * LSX : L * CSX;
};

// PLAIN: no fused operation (op.kind == AXIS_PLAIN), compiled without its branches
template <typename T, int L, int TPL, bool PLAIN>
__global__ void __launch_bounds__(AXIS_THREADS) k_axis_fft(Cx<T>* __restrict__ data, uint64_t Bo, uint64_t Bi,
                                                           uint64_t tiles_i, const Cx<T>* __restrict__ twg,
                                                           int inverse, int shift, int out_neg, T scale,
                                                           int do_scale, AxisOp op, int vec) {
    constexpr int LINES = AXIS_THREADS / TPL;
    constexpr int R = L / TPL;
    using F = LineFFT<T, L, TPL>;
    using G = AxisTile<L, TPL>;
    constexpr int LSX = G::LSX, CSX = G::CSX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T>* buf = reinterpret_cast<Cx<T>*>(smem_raw);
    Cx<T>* tw = buf + G::ELEMS;
    const int t = threadIdx.x;
    const Cx<T> zero = {T(0), T(0)};

    const uint64_t tile = blockIdx.x;
    const bool contig = (Bi == 1);
    // element n of line l: rows [l][n] (pitch LSX) for a contiguous axis,
    // columns [n][l] (pitch CSX) for a strided one, so that the staging copies
    // (consecutive lines of one n) and the transforms both stay conflict-free
    auto slot = [&](int l, int n) { return contig ? l * LSX + n : n * CSX + l; };
    const int ss = contig ? 1 : CSX;  // slot stride along a line
    uint64_t o0 = 0, i0 = 0;
    if (contig) {
        o0 = tile * LINES;
    } else {
        o0 = tile / tiles_i;
        i0 = (tile % tiles_i) * LINES;
    }
    // Staging and write-back walk the tile in steps of AXIS_THREADS elements.
    // Contiguous tiles: element e of the tile is global o0 * L + e.  Strided
    // tiles: a thread keeps one line sl = t % LINES and visits n = sn + TPL j,
    // so its global address advances by TPL * Bi per step.
    const uint64_t g0 = o0 * (uint64_t)L;
    const int sl = t % LINES, sn = t / LINES;
    const bool sl_ok = (i0 + sl) < Bi;
    const uint64_t sg = (o0 * L + sn) * Bi + i0 + sl, gstep = (uint64_t)TPL * Bi;
    auto copy_in = [&](Cx<T>* d, const Cx<T>* src) {
        if constexpr (sizeof(T) == 8)
            cp_async16(d, src);
        else
            cp_async8(d, src);
    };
    // the tile by asynchronous copies, all in flight at once: float pairs of
    // a contiguous tile in 16 bytes (vec: data 16-byte aligned; an even line
    // pitch keeps every pair 16-byte aligned in shared memory), otherwise
    // element by element (a strided tile is transposed into lines); lines
    // past the end are zero-filled
    const bool pairs = sizeof(T) == 4 && LSX % 2 == 0 && contig && vec;
    if (pairs) {
        for (int e = t; e < LINES * L / 2; e += AXIS_THREADS) {
            const int l = (2 * e) / L, n = (2 * e) % L;
            if ((o0 + l) < Bo) {
                cp_async16(buf + l * LSX + n, data + g0 + 2 * e);
            } else {
                buf[l * LSX + n] = zero;
                buf[l * LSX + n + 1] = zero;
            }
        }
    } else if (contig) {
        for (int e = t; e < LINES * L; e += AXIS_THREADS) {
            const int l = e / L, n = e % L;
            if ((o0 + l) < Bo)
                copy_in(buf + l * LSX + n, data + g0 + e);
            else
                buf[l * LSX + n] = zero;
        }
    } else if (sl_ok) {
        const Cx<T>* src = data + sg;
        Cx<T>* d = buf + sn * CSX + sl;
#pragma unroll 4
        for (int j = 0; j < R; ++j, src += gstep, d += TPL * CSX) copy_in(d, src);
    } else {
        for (int j = 0; j < R; ++j) buf[(sn + TPL * j) * CSX + sl] = zero;
    }
    cp_async_commit();
    F::fill_twiddles(tw, twg, t, AXIS_THREADS);
    cp_async_wait<0>();
    __syncthreads();

    const int line = t / TPL, q = t % TPL;
    // global index of element n of this thread's line, and whether the line exists
    const bool line_ok = contig ? (o0 + line) < Bo : (i0 + line) < Bi;
    auto gindex = [&](int n) -> uint64_t {
        return contig ? (o0 + line) * (uint64_t)L + n : (o0 * L + n) * Bi + i0 + line;
    };
    // the constraint's index gi % aux_plane; the arrays of one volume never
    // wrap, and the 64-bit remainder per element is then skipped
    const bool aux_wraps = Bo * (uint64_t)L * Bi > op.aux_plane;
    auto aux_index = [&](uint64_t gi) -> uint64_t { return aux_wraps ? gi % op.aux_plane : gi; };
    Cx<T>* lb = buf + slot(line, 0);  // this line's slots, stride ss
    Cx<T> v[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int n = q + TPL * k;
        v[k] = lb[n * ss];
        if constexpr (!PLAIN) {
            if (op.kind == AXIS_T2_PROLOGUE && line_ok) {
                const uint64_t gi = gindex(n);
                const T sv = static_cast<const T*>(op.aux)[aux_index(gi)];
                v[k] = merge_apply(static_cast<const Cx<T>*>(op.x_in)[gi], space_apply(v[k], sv, op.space_mode),
                                   (T)op.a, (T)op.b);
            }
        }
        if (shift) v[k] = csign(v[k], n);
    }
    Cx<T> o[R];
    if (inverse)
        F::template natural_to_split_flat<true>(v, o, lb, ss, tw, q);
    else
        F::template natural_to_split_flat<false>(v, o, lb, ss, tw, q);
    if constexpr (!PLAIN) {
        if (op.kind == AXIS_DC_ROUNDTRIP || op.kind == AXIS_DCR_ROUNDTRIP) {
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const int f = F::pos(q, i);
                Cx<T> w = o[i];
                if (shift) w = csign(w, f + out_neg);
                if (line_ok) {
                    const uint64_t ai = aux_index(gindex(f));
                    w = (op.kind == AXIS_DC_ROUNDTRIP)
                            ? data_apply_complex(w, static_cast<const Cx<T>*>(op.aux)[ai])
                            : data_apply(w, static_cast<const T*>(op.aux)[ai], op.data_mode);
                }
                if (shift) w = csign(w, f);  // the inverse pass's input flip
                lb[f * ss] = w;
            }
            __syncwarp();
#pragma unroll
            for (int k = 0; k < R; ++k) v[k] = lb[(q + TPL * k) * ss];
            F::template natural_to_split_flat<true>(v, o, lb, ss, tw, q);
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int f = F::pos(q, i);
        Cx<T> w = o[i];
        if (do_scale) w = cscale(w, scale);
        if (shift) w = csign(w, f + out_neg);
        if constexpr (!PLAIN) {
            if (line_ok) {
                if (op.kind == AXIS_SPACE) {
                    w = space_apply(w, static_cast<const T*>(op.aux)[aux_index(gindex(f))], op.space_mode);
                } else if (op.kind == AXIS_T1_EPILOGUE) {
                    const uint64_t gi = gindex(f);
                    w = space_apply(merge_apply(static_cast<const Cx<T>*>(op.x_in)[gi], w, (T)op.a, (T)op.b),
                                    static_cast<const T*>(op.aux)[aux_index(gi)], op.space_mode);
                } else if (op.kind == AXIS_X_EPILOGUE) {
                    const uint64_t gi = gindex(f);
                    Cx<T>* X = static_cast<Cx<T>*>(op.x_in);
                    const Cx<T> x1 =
                        merge_apply(static_cast<const Cx<T>*>(op.t1_in)[gi], X[gi], (T)op.a, (T)op.b);
                    X[gi] = merge_apply(w, x1, (T)op.a2, (T)op.b2);
                }
            }
        }
        lb[f * ss] = w;
    }
    __syncthreads();
    if (pairs) {
        for (int e = t; e < LINES * L / 2; e += AXIS_THREADS) {
            const int l = (2 * e) / L, n = (2 * e) % L;
            if ((o0 + l) < Bo)
                *reinterpret_cast<float4*>(data + g0 + 2 * e) = *reinterpret_cast<const float4*>(buf + l * LSX + n);
        }
    } else if (contig) {
        for (int e = t; e < LINES * L; e += AXIS_THREADS) {
            const int l = e / L, n = e % L;
            if ((o0 + l) < Bo) data[g0 + e] = buf[l * LSX + n];
        }
    } else if (sl_ok) {
        Cx<T>* dst = data + sg;
        const Cx<T>* s = buf + sn * CSX + sl;
#pragma unroll 4
        for (int j = 0; j < R; ++j, dst += gstep, s += TPL * CSX) *dst = *s;
    }
}

template <typename T, int L, int TPL>
cudaError_t axis_fft_t(void* x, uint64_t Bo, uint64_t Bi, bool inverse, bool shift, int out_neg, T scale,
                       bool do_scale, const void* tw, cudaStream_t st, AxisOp op = AxisOp{}) {
    constexpr int LINES = AXIS_THREADS / TPL;
    const size_t smem = sizeof(Cx<T>) * ((size_t)AxisTile<L, TPL>::ELEMS + LineFFT<T, L, TPL>::TW_ENTRIES);
    auto kf = (op.kind == AXIS_PLAIN) ? k_axis_fft<T, L, TPL, true> : k_axis_fft<T, L, TPL, false>;
    cudaError_t e = cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    uint64_t tiles_i = 1, tiles;
    if (Bi == 1) {
        tiles = (Bo + LINES - 1) / LINES;
    } else {
        tiles_i = (Bi + LINES - 1) / LINES;
        tiles = Bo * tiles_i;
    }
    if (tiles == 0) return cudaSuccess;
    if (tiles > 0x7fffffffull) return cudaErrorInvalidValue;
    const int vec = (reinterpret_cast<uintptr_t>(x) & 15u) == 0;
    kf<<<(unsigned)tiles, AXIS_THREADS, smem, st>>>((Cx<T>*)x, Bo, Bi, tiles_i, (const Cx<T>*)tw, inverse ? 1 : 0,
                                                    shift ? 1 : 0, out_neg, scale, do_scale ? 1 : 0, op, vec);
    count_launches();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// one axis, any length: direct DFT, out of place
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_axis_dft(const Cx<T>* __restrict__ in, Cx<T>* __restrict__ out, uint64_t Bo, uint64_t L,
                           uint64_t Bi, const Cx<T>* __restrict__ tw, int inverse, int shift, int out_neg, T scale,
                           int do_scale) {
    const uint64_t total = Bo * L * Bi;
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = idx % Bi;
        const uint64_t f = (idx / Bi) % L;
        const uint64_t o = idx / (Bi * L);
        const Cx<T>* line = in + o * L * Bi + i;
        Cx<T> acc = {T(0), T(0)};
        uint64_t w = 0;
        for (uint64_t n = 0; n < L; ++n) {
            Cx<T> a = line[n * Bi];
            if (shift && (n & 1)) a = cneg(a);
            const Cx<T> t = inverse ? cmulc(a, tw[w]) : cmul(a, tw[w]);
            acc = cadd(acc, t);
            w += f;
            if (w >= L) w -= L;
        }
        if (do_scale) acc = cscale(acc, scale);
        if (shift) acc = csign(acc, (int)(f & 1) + out_neg);
        out[idx] = acc;
    }
}

template <typename T>
cudaError_t axis_dft_t(void* x, void* work, uint64_t Bo, uint64_t L, uint64_t Bi, bool inverse, bool shift,
                       int out_neg, T scale, bool do_scale, const void* tw, cudaStream_t st) {
    const uint64_t total = Bo * L * Bi;
    if (total == 0) return cudaSuccess;
    k_axis_dft<T><<<ew_grid(total, 256), 256, 0, st>>>((const Cx<T>*)x, (Cx<T>*)work, Bo, L, Bi,
                                                       (const Cx<T>*)tw, inverse ? 1 : 0, shift ? 1 : 0, out_neg,
                                                       scale, do_scale ? 1 : 0);
    count_launches();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(x, work, total * sizeof(Cx<T>), cudaMemcpyDeviceToDevice, st);
}

bool is_pow2(uint64_t n) { return n > 0 && (n & (n - 1)) == 0; }

template <typename T>
cudaError_t axis_pass(void* x, void* work, uint64_t Bo, uint64_t L, uint64_t Bi, bool inverse, T scale,
                      bool do_scale, const void* tw, cudaStream_t st, AxisOp op = AxisOp{}) {
    const int out_neg = (int)((L / 2) & 1);  // s_a = (-1)^(L/2)
    if (L == 1) {
        if (!do_scale) return cudaSuccess;
        return launch_scale(sizeof(T) == 8, x, (double)scale, Bo * Bi, st);
    }
    if (!is_pow2(L) || L > 1024) return axis_dft_t<T>(x, work, Bo, L, Bi, inverse, true, out_neg, scale, do_scale, tw, st);
    switch (L) {
        case 2: return axis_fft_t<T, 2, 1>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        case 4: return axis_fft_t<T, 4, 1>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        case 8: return axis_fft_t<T, 8, 1>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        case 16: return axis_fft_t<T, 16, 1>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        case 32: return axis_fft_t<T, 32, 1>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        case 64: return axis_fft_t<T, 64, 4>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        case 128: return axis_fft_t<T, 128, 4>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        // 256 and 512: 16 and 32 threads per line, the split of the fused line
        // passes (line_pass.cuh LineGeom), so those round exactly like these calls
        case 256: return axis_fft_t<T, 256, 16>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        case 512: return axis_fft_t<T, 512, 32>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        case 1024: return axis_fft_t<T, 1024, 32>(x, Bo, Bi, inverse, true, out_neg, scale, do_scale, tw, st, op);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t fft2d_t(void* x, uint64_t M, uint64_t N, uint64_t batch, bool inverse, T scale, const void* tw_m,
                    const void* tw_n, void* work, cudaStream_t st) {
    if (M == N && fft2d_single_cta(sizeof(T) == 8, M, N)) {
        const int s_neg = (int)(((M / 2) + (N / 2)) & 1);
        switch (M) {
            case 32: return plane_fft<T, 32>(x, batch, inverse, scale, s_neg, tw_m, st);
            case 64: return plane_fft<T, 64>(x, batch, inverse, scale, s_neg, tw_m, st);
            case 128:
                if constexpr (sizeof(T) == 4) return plane_fft<T, 128>(x, batch, inverse, scale, s_neg, tw_m, st);
                break;
            default: break;
        }
    }
    cudaError_t e;
    if (!inverse) {
        if ((e = axis_pass<T>(x, work, batch * M, N, 1, false, scale, false, tw_n, st)) != cudaSuccess) return e;
        return axis_pass<T>(x, work, batch, M, N, false, scale, false, tw_m, st);
    }
    if ((e = axis_pass<T>(x, work, batch, M, N, true, scale, false, tw_m, st)) != cudaSuccess) return e;
    return axis_pass<T>(x, work, batch * M, N, 1, true, scale, true, tw_n, st);
}

template <typename T>
cudaError_t fft3d_t(void* x, uint64_t M, uint64_t N, uint64_t L, uint64_t batch, bool inverse, T scale,
                    const void* tw_m, const void* tw_n, const void* tw_l, void* work, cudaStream_t st) {
    cudaError_t e;
    if (!inverse) {
        if ((e = axis_pass<T>(x, work, batch * L * M, N, 1, false, scale, false, tw_n, st)) != cudaSuccess) return e;
        if ((e = axis_pass<T>(x, work, batch * L, M, N, false, scale, false, tw_m, st)) != cudaSuccess) return e;
        return axis_pass<T>(x, work, batch, L, M * N, false, scale, false, tw_l, st);
    }
    if ((e = axis_pass<T>(x, work, batch, L, M * N, true, scale, false, tw_l, st)) != cudaSuccess) return e;
    if ((e = axis_pass<T>(x, work, batch * L, M, N, true, scale, false, tw_m, st)) != cudaSuccess) return e;
    return axis_pass<T>(x, work, batch * L * M, N, 1, true, scale, true, tw_n, st);
}

// iters x [Forward3D; DataConstraint(C); Backward3D; SpaceConstraint(S)] as
// five axis passes per iteration (x, y forward; z forward + constraint +
// inverse; y inverse; x inverse + SpaceConstraint), the per-call passes'
// arithmetic in the same order
template <typename T>
cudaError_t constraint3d_t(void* x, const void* C, const void* S, uint64_t M, uint64_t N, uint64_t L, uint64_t batch,
                           int iters, int space_mode, T scale, const void* tw_m, const void* tw_n, const void* tw_l,
                           void* work, cudaStream_t st) {
    const uint64_t plane = M * N * L;
    AxisOp dc;
    dc.kind = AXIS_DC_ROUNDTRIP;
    dc.aux = C;
    dc.aux_plane = plane;
    AxisOp sc;
    sc.kind = AXIS_SPACE;
    sc.aux = S;
    sc.aux_plane = plane;
    sc.space_mode = space_mode;
    cudaError_t e;
    for (int it = 0; it < iters; ++it) {
        if ((e = axis_pass<T>(x, work, batch * L * M, N, 1, false, scale, false, tw_n, st)) != cudaSuccess) return e;
        if ((e = axis_pass<T>(x, work, batch * L, M, N, false, scale, false, tw_m, st)) != cudaSuccess) return e;
        if ((e = axis_pass<T>(x, work, batch, L, M * N, false, scale, false, tw_l, st, dc)) != cudaSuccess) return e;
        if ((e = axis_pass<T>(x, work, batch * L, M, N, true, scale, false, tw_m, st)) != cudaSuccess) return e;
        if ((e = axis_pass<T>(x, work, batch * L * M, N, 1, true, scale, true, tw_n, st, sc)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// the difference-map iteration (src/CPRA_MKL.cpp:94-110, here with the 3D
// transforms: src/CONV_MKL.cpp:37-88), `iters` times, as ten axis passes:
// t1's projection (x, y forward; z forward + modulus + inverse; y inverse; x
// inverse + merge with x + SpaceConstraint), then t2's (x forward from
// a2*x + b2*S(t2); y; z; y; x inverse + the merges into x)
template <typename T>
cudaError_t dm3d_t(const DmArgs& a, T scale, const void* tw_m, const void* tw_n, const void* tw_l, void* work,
                   cudaStream_t st) {
    const uint64_t M = a.M, N = a.N, L = a.L, batch = a.batch, plane = M * N * L;
    AxisOp dc;
    dc.kind = AXIS_DCR_ROUNDTRIP;
    dc.aux = a.A;
    dc.aux_plane = plane;
    dc.data_mode = a.data_mode;
    AxisOp e1;
    e1.kind = AXIS_T1_EPILOGUE;
    e1.aux = a.S;
    e1.aux_plane = plane;
    e1.space_mode = a.space_mode;
    e1.x_in = a.x;
    e1.a = a.c.a1;
    e1.b = a.c.b1;
    AxisOp p2;
    p2.kind = AXIS_T2_PROLOGUE;
    p2.aux = a.S;
    p2.aux_plane = plane;
    p2.space_mode = a.space_mode;
    p2.x_in = a.x;
    p2.a = a.c.a2;
    p2.b = a.c.b2;
    AxisOp ex;
    ex.kind = AXIS_X_EPILOGUE;
    ex.x_in = a.x;
    ex.t1_in = a.t1;
    ex.a = a.c.a3;
    ex.b = a.c.b3;
    ex.a2 = a.c.a4;
    ex.b2 = a.c.b4;
    cudaError_t e;
    auto project = [&](void* v, AxisOp first, AxisOp last) -> cudaError_t {
        cudaError_t r;
        if ((r = axis_pass<T>(v, work, batch * L * M, N, 1, false, scale, false, tw_n, st, first)) != cudaSuccess)
            return r;
        if ((r = axis_pass<T>(v, work, batch * L, M, N, false, scale, false, tw_m, st)) != cudaSuccess) return r;
        if ((r = axis_pass<T>(v, work, batch, L, M * N, false, scale, false, tw_l, st, dc)) != cudaSuccess) return r;
        if ((r = axis_pass<T>(v, work, batch * L, M, N, true, scale, false, tw_m, st)) != cudaSuccess) return r;
        return axis_pass<T>(v, work, batch * L * M, N, 1, true, scale, true, tw_n, st, last);
    };
    for (int it = 0; it < a.iters; ++it) {
        if ((e = project(a.t1, AxisOp{}, e1)) != cudaSuccess) return e;
        if ((e = project(a.t2, p2, ex)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_dm3d_iterations(bool dbl, const DmArgs& a, double scale, const void* tw_m, const void* tw_n,
                                   const void* tw_l, void* work, cudaStream_t st) {
    if (!constraint3d_fused_supported(a.M, a.N, a.L)) return cudaErrorInvalidValue;
    if (a.batch == 0 || a.iters <= 0) return cudaSuccess;
    return dbl ? dm3d_t<double>(a, scale, tw_m, tw_n, tw_l, work, st)
               : dm3d_t<float>(a, (float)scale, tw_m, tw_n, tw_l, work, st);
}

bool constraint3d_fused_supported(uint64_t M, uint64_t N, uint64_t L) {
    auto p2 = [](uint64_t v) { return v >= 2 && (v & (v - 1)) == 0 && v <= 1024; };
    return p2(M) && p2(N) && p2(L);
}

cudaError_t launch_constraint3d(bool dbl, void* x, const void* C, const void* S, uint64_t M, uint64_t N, uint64_t L,
                                uint64_t batch, int iters, int space_mode, double scale, const void* tw_m,
                                const void* tw_n, const void* tw_l, void* work, cudaStream_t st) {
    if (!constraint3d_fused_supported(M, N, L)) return cudaErrorInvalidValue;
    if (batch == 0 || iters <= 0) return cudaSuccess;
    return dbl ? constraint3d_t<double>(x, C, S, M, N, L, batch, iters, space_mode, scale, tw_m, tw_n, tw_l, work, st)
               : constraint3d_t<float>(x, C, S, M, N, L, batch, iters, space_mode, (float)scale, tw_m, tw_n, tw_l,
                                       work, st);
}

bool fft2d_single_cta(bool dbl, uint64_t M, uint64_t N) {
    if (M != N) return false;
    if (dbl) return M == 32 || M == 64;
    return M == 32 || M == 64 || M == 128;
}

bool fft_length_supported(uint64_t L) { return L >= 1 && L <= 4096 && (L == 1 || (L % 2) == 0); }

cudaError_t launch_fft2d(bool dbl, void* x, uint64_t M, uint64_t N, uint64_t batch, bool inverse, double scale,
                         const void* tw_m, const void* tw_n, void* work, cudaStream_t st) {
    if (batch == 0) return cudaSuccess;
    return dbl ? fft2d_t<double>(x, M, N, batch, inverse, scale, tw_m, tw_n, work, st)
               : fft2d_t<float>(x, M, N, batch, inverse, (float)scale, tw_m, tw_n, work, st);
}

cudaError_t launch_fft3d(bool dbl, void* x, uint64_t M, uint64_t N, uint64_t L, uint64_t batch, bool inverse,
                         double scale, const void* tw_m, const void* tw_n, const void* tw_l, void* work,
                         cudaStream_t st) {
    if (batch == 0) return cudaSuccess;
    return dbl ? fft3d_t<double>(x, M, N, L, batch, inverse, scale, tw_m, tw_n, tw_l, work, st)
               : fft3d_t<float>(x, M, N, L, batch, inverse, (float)scale, tw_m, tw_n, tw_l, work, st);
}

}  // namespace cpra_b200
