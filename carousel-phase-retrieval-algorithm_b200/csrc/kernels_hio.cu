// Hybrid input-output iterations with shrinkwrap support updates, fused: one
// CTA per pattern, `iters` iterations per launch.  Project-defined (the
// reference's "shrinkwrap" drivers run the difference map with a fixed
// support, src/CPRA_MKL.cpp:94-110; it has no HIO and no support update).
//
// Per iteration, with y = P_M(x) = Backward2D(DataConstraint(Forward2D(x)))
// (the reference operators' composition, modulus plane A):
//   x <- y            where the pixel is in the support (and Re y >= 0 with
//                     positivity on),
//   x <- x - beta*y   elsewhere.
// Every `sw_every` iterations the support becomes { v > threshold * max v }
// with v = |x| blurred by a normalised periodic Gaussian (circular
// convolution, evaluated exactly through the DFT: the separable transfer
// function g(f_row) g(f_col) is a table per update, sigma moving linearly from
// sigma_start at the first update to sigma_end at the last).
//
// On chip: the plane buffer of the transforms, A and the support (a bit mask)
// in shared memory.  Each thread keeps the x values of its own positions in
// registers for the next iteration's forward transform and holds the first
// half of them through the transforms, so only the second half goes through
// L2 (written and read once per iteration).  The first half is written before
// each support update, whose blur reuses those registers (x is read back in
// full after it), and after the last iteration.  Optionally the kernel also
// writes the estimate S (.) P_M(x) of the final x.
//
// Two more forms of the same iteration follow: k_hio_tm (128 x 128, 1024
// threads, x in the SM's tensor memory) and k_hio_cl (128 x 128 and
// 256 x 256 patterns spread over a thread-block cluster, for batches that
// would leave SMs idle with one CTA per pattern).
#include "cpra_internal.h"
#include "fft2d_cta.cuh"
#include "ops_ew.cuh"
#include "cluster.cuh"
#include "tmem.cuh"

namespace cpra_b200 {

namespace {

struct HioDev {
    Cx<float>* x;
    Cx<float>* est;  // optional: S (.) P_M(x) after the last iteration
    const float* A;
    uint64_t a_stride;
    float* S;
    uint64_t s_stride;
    const Cx<float>* tw;
    const float* blur;  // [updates][L]: g at the frequency of each (D-shifted) row/column index
    int* err;           // cluster kernel: set to 1 when a wait for a peer's data ran out
    int withhold;       // cluster kernel, failure test: CTA 0 sends none of its first row blocks
    float scale, beta, thresh;
    int iters, sw_every, positivity, data_mode;
};

template <int L>
struct HioPlan {
    using P = Plane<float, L>;
    static constexpr int AP = L + 8;
    static constexpr int MASK_WORDS = L * L / 32;
    static constexpr int WARPS = P::NT / 32;
    static constexpr size_t a_bytes() { return sizeof(float) * (size_t)L * AP; }
    static constexpr size_t smem_bytes() {
        return P::buf_bytes() + a_bytes() + P::tw_bytes() + sizeof(uint32_t) * MASK_WORDS + sizeof(float) * L +
               sizeof(float) * WARPS;
    }
};

// column forward transform, a per-frequency operation, column inverse transform
template <class P, class Op>
__device__ __forceinline__ void spectral_columns_t(Cx<float>* buf, const Cx<float>* tw, int c, int q, Op op) {
    Cx<float> o[P::J][P::TPL];
    P::template col_from_buf<false>(o, buf, tw, c, q);
#pragma unroll
    for (int j = 0; j < P::J; ++j)
#pragma unroll
        for (int s = 0; s < P::TPL; ++s) o[j][s] = op(o[j][s], P::split_pos(q, j, s), c);
    P::template col_to_buf<true>(o, buf, tw, c, q);
}
template <int L, class Op>
__device__ __forceinline__ void spectral_columns(Cx<float>* buf, const Cx<float>* tw, int c, int q, Op op) {
    using P = Plane<float, L>;
    Cx<float> o[P::J][P::TPL];
    P::template col_from_buf<false>(o, buf, tw, c, q);
#pragma unroll
    for (int j = 0; j < P::J; ++j)
#pragma unroll
        for (int s = 0; s < P::TPL; ++s) o[j][s] = op(o[j][s], P::split_pos(q, j, s), c);
    P::template col_to_buf<true>(o, buf, tw, c, q);
}

// DMODE: the DataConstraint mode; POS: positivity inside the support.  Both
// fixed at compile time so that each instantiation carries only its own
// arithmetic.  At 64^2 three CTAs share an SM (at most 80 registers, no
// spills; left unbounded the kernel takes 170 and one CTA per SM).
template <int L, int DMODE, bool POS>
__global__ void __launch_bounds__(4 * L, (L == 64) ? 3 : 1) k_hio(const HioDev p) {
    using P = Plane<float, L>;
    using H = HioPlan<L>;
    constexpr int J = P::J, TPL = P::TPL, AP = H::AP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* buf = reinterpret_cast<Cx<float>*>(smem_raw);
    float* As = reinterpret_cast<float*>(smem_raw + P::buf_bytes());
    Cx<float>* tw = reinterpret_cast<Cx<float>*>(smem_raw + P::buf_bytes() + H::a_bytes());
    uint32_t* mask = reinterpret_cast<uint32_t*>(smem_raw + P::buf_bytes() + H::a_bytes() + P::tw_bytes());
    float* gt = reinterpret_cast<float*>(mask + H::MASK_WORDS);
    float* red = gt + L;
    const int t = threadIdx.x, line = t >> 2, q = t & 3;
    P::F::fill_twiddles(tw, p.tw, t, P::NT);
    Cx<float>* __restrict__ X = p.x + (size_t)blockIdx.x * L * L;
    const float* __restrict__ A = p.A + blockIdx.x * p.a_stride;
    float* __restrict__ S = p.S + blockIdx.x * p.s_stride;
    for (int i = t; i < L * L; i += P::NT) As[(i / L) * AP + (i % L)] = A[i];
    for (int i = t; i < L * L; i += P::NT) {
        const unsigned in = __ballot_sync(0xffffffffu, S[i] > 0.5f);
        if ((i & 31) == 0) mask[i >> 5] = in;
    }
    auto at = [&](int j, int s) { return line * L + P::split_pos(q, j, s); };
    const bool neg = ((line + q) & 1) != 0;
    auto sgn = [&](Cx<float> z) { return neg ? Cx<float>{-z.x, -z.y} : z; };
    auto inside = [&](int idx) { return (mask[idx >> 5] >> (idx & 31)) & 1u; };
    __syncthreads();

    int update = 0;
    // o: this thread's x values at the top of each iteration
    Cx<float> o[J][TPL];
    auto load_x = [&]() {
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) o[j][s] = X[at(j, s)];
    };
    load_x();
    for (int it = 0; it < p.iters; ++it) {
        // xh: the first J/2 split columns of x, kept through the transforms
        Cx<float> xh[J / 2][TPL];
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                if (j < J / 2) xh[j][s] = o[j][s];
                o[j][s] = sgn(o[j][s]);
            }
        P::template rows_split_to_buf<false>(o, buf, tw, line, q);
        __syncthreads();
        spectral_columns<L>(buf, tw, line, q, [&](Cx<float> z, int f, int c) {
            return data_apply(z, As[f * AP + c], DMODE);
        });
        __syncthreads();
        P::template row_from_buf<true>(o, buf, tw, line, q);
        const bool update_next = p.sw_every > 0 && p.blur && (it + 1) % p.sw_every == 0;
        // the first half of x lives in registers from here to the next
        // update; it goes to memory only before a support update (whose blur
        // reuses the registers) and after the last iteration
        const bool store_all = update_next || it + 1 == p.iters;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                const int idx = at(j, s);
                const Cx<float> y = sgn(cscale(o[j][s], p.scale));
                const Cx<float> xv = (j < J / 2) ? xh[j][s] : X[idx];
                const bool keep = inside(idx) && (!POS || y.x >= 0.0f);
                const Cx<float> xn = keep ? y : merge_apply(y, xv, -p.beta, 1.0f);
                if (j >= J / 2 || store_all) X[idx] = xn;
                o[j][s] = xn;
            }
        if (!update_next) continue;

        // ---- shrinkwrap: v = |x| blurred, support = { v > thresh * max v } ----
        if (t < L) gt[t] = p.blur[(size_t)update * L + t];
        ++update;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                const Cx<float> z = o[j][s];
                o[j][s] = sgn(Cx<float>{sqrtf(fmaf(z.x, z.x, z.y * z.y)), 0.0f});
            }
        P::template rows_split_to_buf<false>(o, buf, tw, line, q);
        __syncthreads();
        spectral_columns<L>(buf, tw, line, q, [&](Cx<float> z, int f, int c) { return cscale(z, gt[f] * gt[c]); });
        __syncthreads();
        P::template row_from_buf<true>(o, buf, tw, line, q);
        float vmax = -INFINITY;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                o[j][s].x = sgn(cscale(o[j][s], p.scale)).x;
                vmax = fmaxf(vmax, o[j][s].x);
            }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
        if ((t & 31) == 0) red[t >> 5] = vmax;
        __syncthreads();
        float m = red[0];
        for (int w = 1; w < H::WARPS; ++w) m = fmaxf(m, red[w]);
        const float thr = p.thresh * m;
        // this row's mask words are read and written only by its four threads
        for (int w = q; w < L / 32; w += TPL) mask[line * (L / 32) + w] = 0u;
        __syncwarp();
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s)
                if (o[j][s].x > thr) {
                    const int idx = at(j, s);
                    atomicOr(&mask[idx >> 5], 1u << (idx & 31));
                }
        __syncthreads();  // red[] is reused by the next update
        load_x();         // the blur overwrote o
    }
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int s = 0; s < TPL; ++s) S[at(j, s)] = inside(at(j, s)) ? 1.0f : 0.0f;
    if (!p.est) return;
    // the estimate: the modulus projection of the final x, restricted to the support
    Cx<float>* __restrict__ E = p.est + (size_t)blockIdx.x * L * L;
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int s = 0; s < TPL; ++s) o[j][s] = sgn(X[at(j, s)]);
    P::template rows_split_to_buf<false>(o, buf, tw, line, q);
    __syncthreads();
    spectral_columns<L>(buf, tw, line, q, [&](Cx<float> z, int f, int c) {
        return data_apply(z, As[f * AP + c], DMODE);
    });
    __syncthreads();
    P::template row_from_buf<true>(o, buf, tw, line, q);
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int s = 0; s < TPL; ++s) {
            const int idx = at(j, s);
            E[idx] = inside(idx) ? sgn(cscale(o[j][s], p.scale)) : Cx<float>{0.0f, 0.0f};
        }
}

// The 128 x 128 kernel with x in tensor memory and 8 threads per line.
//
// A thread reads and writes x only at its own row's 16 split positions, and
// the support only at the same pixels, so both are thread-private: x lives in
// the SM's tensor memory for the whole launch (warp w's threads own lane
// 32*(w % 4) + lane id, columns (w / 4)*32 .. +31, element (j, s) at
// 2*(8j + s)), the support of the thread's 16 pixels in one register of bits.
// Registers then hold only the 16 transform values, the CTA runs 1024 threads
// (32 warps per SM), and global memory is touched when the launch starts (x,
// A, S) and after the last iteration (x, S, the estimate).  The shrinkwrap
// blur reads x back from tensor memory.  The transforms split each line over
// 8 threads as the float 128 x 128 plane kernels do (plane_tpl); the
// iteration is k_hio's.
template <int DMODE, bool POS>
__global__ void __launch_bounds__(1024, 1) k_hio_tm(const HioDev p) {
    constexpr int L = 128;
    using P = Plane<float, L, plane_tpl<float, L>()>;
    constexpr int J = P::J, TPL = P::TPL, AP = L + 4, WARPS = P::NT / 32;
    static_assert(TPL == 8 && J == 2 && P::NT == 1024, "two 8-value groups per thread, 32 warps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t tm_base;
    Cx<float>* buf = reinterpret_cast<Cx<float>*>(smem_raw);
    float* As = reinterpret_cast<float*>(smem_raw + P::buf_bytes());
    Cx<float>* tw = reinterpret_cast<Cx<float>*>(smem_raw + P::buf_bytes() + sizeof(float) * L * AP);
    float* gt = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(tw) + P::tw_bytes());
    float* red = gt + L;
    const int t = threadIdx.x, row = P::row_of(t), col = P::col_of(t), q = P::rank_of(t), warp = t >> 5;
    if (warp == 0) tm_alloc(&tm_base, 256);
    P::F::fill_twiddles(tw, p.tw, t, P::NT);
    Cx<float>* __restrict__ X = p.x + (size_t)blockIdx.x * L * L;
    const float* __restrict__ A = p.A + blockIdx.x * p.a_stride;
    float* __restrict__ S = p.S + blockIdx.x * p.s_stride;
    for (int i = t; i < L * L; i += P::NT) As[(i / L) * AP + (i % L)] = A[i];
    auto at = [&](int j, int s) { return row * L + P::split_pos(q, j, s); };
    const bool neg = ((row + q) & 1) != 0;
    auto sgn = [&](Cx<float> z) { return neg ? Cx<float>{-z.x, -z.y} : z; };
    // the support of this thread's pixels: bit 8j + s
    uint32_t in_bits = 0;
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int s = 0; s < TPL; ++s) in_bits |= (S[at(j, s)] > 0.5f ? 1u : 0u) << (TPL * j + s);
    auto inside = [&](int j, int s) { return (in_bits >> (TPL * j + s)) & 1u; };
    tm_fence_before_sync();
    __syncthreads();
    tm_fence_after_sync();
    const uint32_t xa = tm_lane_addr(tm_base, warp, (warp >> 2) * 32);
    Cx<float> o[J][TPL];
    // x into tensor memory (group g = 2j + h: elements s in [4h, 4h + 4))
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            Cx<float> xs[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                xs[u] = X[at(j, 4 * h + u)];
                o[j][4 * h + u] = xs[u];
            }
            tm_st4(xa + 8 * (2 * j + h), xs);
        }
    int update = 0;
    for (int it = 0; it < p.iters; ++it) {
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) o[j][s] = sgn(o[j][s]);
        P::template rows_split_to_buf<false>(o, buf, tw, row, q);
        __syncthreads();
        spectral_columns_t<P>(buf, tw, col, q, [&](Cx<float> z, int f, int c) {
            return data_apply(z, As[f * AP + c], DMODE);
        });
        __syncthreads();
        P::template row_from_buf<true>(o, buf, tw, row, q);
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                Cx<float> xr[4];
                tm_ld4(xa + 8 * (2 * j + h), xr);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int s = 4 * h + u;
                    const Cx<float> y = sgn(cscale(o[j][s], p.scale));
                    const bool keep = inside(j, s) && (!POS || y.x >= 0.0f);
                    xr[u] = keep ? y : merge_apply(y, xr[u], -p.beta, 1.0f);
                    o[j][s] = xr[u];
                }
                tm_st4(xa + 8 * (2 * j + h), xr);
            }
        const bool update_next = p.sw_every > 0 && p.blur && (it + 1) % p.sw_every == 0;
        if (!update_next) continue;

        // ---- shrinkwrap: v = |x| blurred, support = { v > thresh * max v } ----
        if (t < L) gt[t] = p.blur[(size_t)update * L + t];
        ++update;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                const Cx<float> z = o[j][s];
                o[j][s] = sgn(Cx<float>{sqrtf(fmaf(z.x, z.x, z.y * z.y)), 0.0f});
            }
        P::template rows_split_to_buf<false>(o, buf, tw, row, q);
        __syncthreads();
        spectral_columns_t<P>(buf, tw, col, q, [&](Cx<float> z, int f, int c) { return cscale(z, gt[f] * gt[c]); });
        __syncthreads();
        P::template row_from_buf<true>(o, buf, tw, row, q);
        float vmax = -INFINITY;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                o[j][s].x = sgn(cscale(o[j][s], p.scale)).x;
                vmax = fmaxf(vmax, o[j][s].x);
            }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
        if ((t & 31) == 0) red[t >> 5] = vmax;
        __syncthreads();
        float m = red[0];
        for (int w = 1; w < WARPS; ++w) m = fmaxf(m, red[w]);
        const float thr = p.thresh * m;
        in_bits = 0;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) in_bits |= (o[j][s].x > thr ? 1u : 0u) << (TPL * j + s);
        __syncthreads();  // red[] is reused by the next update
        // the blur overwrote o: x again from tensor memory
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                Cx<float> xr[4];
                tm_ld4(xa + 8 * (2 * j + h), xr);
#pragma unroll
                for (int u = 0; u < 4; ++u) o[j][4 * h + u] = xr[u];
            }
    }
    // x and the support out (the addresses again from the block index, so
    // that no pointer stays in a register through the iterations)
    const unsigned b = cta_index();
    Cx<float>* __restrict__ Xo = p.x + (size_t)b * L * L;
    float* __restrict__ So = p.S + b * p.s_stride;
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int s = 0; s < TPL; ++s) {
            Xo[at(j, s)] = o[j][s];
            So[at(j, s)] = inside(j, s) ? 1.0f : 0.0f;
        }
    if (p.est) {
        // the estimate: the modulus projection of the final x, restricted to the support
        Cx<float>* __restrict__ E = p.est + (size_t)b * L * L;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) o[j][s] = sgn(o[j][s]);
        P::template rows_split_to_buf<false>(o, buf, tw, row, q);
        __syncthreads();
        spectral_columns_t<P>(buf, tw, col, q, [&](Cx<float> z, int f, int c) {
            return data_apply(z, As[f * AP + c], DMODE);
        });
        __syncthreads();
        P::template row_from_buf<true>(o, buf, tw, row, q);
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s)
                E[at(j, s)] = inside(j, s) ? sgn(cscale(o[j][s], p.scale)) : Cx<float>{0.0f, 0.0f};
    }
    tm_wait_st();
    tm_fence_before_sync();
    __syncthreads();
    tm_fence_after_sync();
    if (warp == 0) tm_free(tm_base, 256);
}

size_t hio_tm_smem_bytes() {
    using P = Plane<float, 128, plane_tpl<float, 128>()>;
    return P::buf_bytes() + sizeof(float) * 128 * (128 + 4) + P::tw_bytes() + sizeof(float) * 128 +
           sizeof(float) * (P::NT / 32);
}

// ---- one pattern over a thread-block cluster of CL CTAs ----------------------------------
//
// CTA rank r of a pattern's cluster owns rows r*RPC .. r*RPC + RPC - 1 in the
// row phases and the same range of columns in the column phase (RPC = L/CL).
// A line is TPL threads (8 at 128, 16 at 256) with R = L/TPL values each.
// Per transform of the plane:
//   row phase     each row, from registers, through its row DFT into the
//                 row buffer (scratch and result: the row's own slots); the
//                 row's RPC-element block of each CTA's columns goes to that
//                 CTA's column buffer in one bulk copy
//   column phase  (once every CTA's blocks have arrived) each owned column
//                 through the column DFT, the per-frequency operation (the
//                 modulus projection or the shrinkwrap blur), the inverse
//                 column DFT, back into the column buffer; the block of each
//                 CTA's rows goes to that CTA's row buffer, one bulk copy per
//                 row
//   row phase     (once every block has arrived) each row through the
//                 inverse row DFT into registers, then the HIO update of x.
// Arrivals are counted in bytes on one mbarrier per buffer, armed for the
// next phase as soon as the current one completes (no data of the next phase
// can be sent before this CTA sends its own part of the current one).  A
// phase whose bytes have not arrived within a second sets the launch's
// error word; the CTA then stops waiting and sending, runs to the end and
// waits once more, bounded, for what is still in flight.  An iteration thus
// moves the plane twice between the SMs' shared memories by the copy
// engines and never through L2; global memory is read when the launch starts
// and written after the last iteration.  The shrinkwrap maximum is
// exchanged with remote stores and a cluster barrier (one value per CTA).
// The line transforms, their scratch layout and every per-element step are
// those of the one-CTA kernels of the same split (k_hio_tm at 128), in the
// same order, so the results are the same bits for any cluster size.
//
// Shared memory: the two mbarriers; the row buffer [RPC][LS] (LS = L + 2;
// the rows of a half-warp 4 apart at TPL 8, so its slots fall on distinct
// bank pairs); the column buffer [L][CP], row-major over the owned columns
// (CP = RPC + 2: a half-warp's two columns and 8 ranks on distinct bank
// pairs, at TPL 16 with the two columns interleaved lane by lane; rows
// 16-byte aligned for the copies); A of the owned
// columns, column-major (pitch ACP); twiddles; a blur table row; maxima.
template <int L, int CL>
struct ClGeom {
    static constexpr int TPL = (L <= 128) ? 8 : 16;
    using F = LineFFT<float, L, TPL>;
    static constexpr int R = L / TPL, J = F::J;
    static constexpr int RPC = L / CL;  // rows (and columns) per CTA
    static constexpr int NT = RPC * TPL;
    static constexpr int LS = L + 2;
    static constexpr int CP = RPC + 2;
    static constexpr int ACP = (TPL == 8) ? L + 8 : L + 16;
    static constexpr int WARPS = NT / 32;
    static constexpr uint32_t BLOCK_BYTES = RPC * sizeof(Cx<float>);         // one copy
    static constexpr uint32_t PHASE_BYTES = (uint32_t)RPC * L * sizeof(Cx<float>);  // a buffer's arrivals
    static_assert(R == 16 && !F::HALF, "16 values per thread");
    static_assert(TPL == 16 || NT % 128 == 0, "TPL 8: rows in groups of 16 per 128 threads");
    static_assert(NT <= 1024 && NT >= L && CL <= TPL, "copy issuers: L threads, CL ranks per row");
    static_assert(BLOCK_BYTES % 16 == 0 && (LS * sizeof(Cx<float>)) % 16 == 0 && (CP * sizeof(Cx<float>)) % 16 == 0,
                  "16-byte copies");
    static constexpr size_t rbuf_off() { return 16; }
    static constexpr size_t cbuf_off() { return rbuf_off() + sizeof(Cx<float>) * (size_t)RPC * LS; }
    static constexpr size_t a_off() { return cbuf_off() + sizeof(Cx<float>) * (size_t)L * CP; }
    static constexpr size_t tw_off() { return a_off() + sizeof(float) * (size_t)RPC * ACP; }
    static constexpr size_t smem_bytes() {
        return tw_off() + sizeof(Cx<float>) * F::TW_ENTRIES + sizeof(float) * (L + WARPS + CL);
    }
    // the row of thread t in the row phases
    __device__ __forceinline__ static int row_of(int t) {
        if constexpr (TPL == 8)
            return ((t >> 7) << 4) + ((t >> 5) & 3) + 4 * ((t >> 3) & 3);
        else
            return t / TPL;
    }
    // the column of thread t in the column phase, and its rank there: at
    // TPL 16 a warp holds two columns interleaved lane by lane, so a
    // half-warp reads 8 ranks of two columns, 16 distinct bank pairs at the
    // even pitch CP (one column of 16 ranks per half-warp would collide 2-way)
    __device__ __forceinline__ static int col_of(int t) {
        if constexpr (TPL == 16)
            return 2 * (t >> 5) + (t & 1);
        else
            return t / TPL;
    }
    __device__ __forceinline__ static int col_rank(int t) {
        if constexpr (TPL == 16)
            return (t & 31) >> 1;
        else
            return t % TPL;
    }
};

// a second: far above any phase of a healthy launch
constexpr uint64_t CLUSTER_WAIT_NS = 1000000000ull;

template <int L, int CL, int DMODE, bool POS>
__global__ void __launch_bounds__(ClGeom<L, CL>::NT, 1) k_hio_cl(const HioDev p) {
    using G = ClGeom<L, CL>;
    using F = typename G::F;
    constexpr int J = G::J, TPL = G::TPL, R = G::R, RPC = G::RPC, LS = G::LS, CP = G::CP, ACP = G::ACP,
                  NT = G::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* rbuf = reinterpret_cast<Cx<float>*>(smem_raw + G::rbuf_off());
    Cx<float>* cbuf = reinterpret_cast<Cx<float>*>(smem_raw + G::cbuf_off());
    float* Ac = reinterpret_cast<float*>(smem_raw + G::a_off());
    Cx<float>* tw = reinterpret_cast<Cx<float>*>(smem_raw + G::tw_off());
    float* gt = reinterpret_cast<float*>(tw + F::TW_ENTRIES);
    float* red = gt + L;           // [WARPS] this CTA's warp maxima
    float* cmax = red + G::WARPS;  // [CL] every CTA's maximum
    const int t = threadIdx.x, q = t % TPL, warp = t >> 5;
    const int row = G::row_of(t);  // this CTA's row in the row phases
    const int cl = G::col_of(t);   // this CTA's column in the column phase
    const int qc = G::col_rank(t);  // and the thread's rank in it
    const int rank = (int)cluster_ctarank();
    const int grow = rank * RPC + row, gcol = rank * RPC + cl;
    const uint32_t base = smem_addr_u32(smem_raw);
    const uint32_t mb_r = base, mb_c = base + 8;  // arrivals into the row / the column buffer
    const uint32_t rb = base + (uint32_t)G::rbuf_off(), cb = base + (uint32_t)G::cbuf_off();
    const uint32_t cm = smem_addr_u32(cmax);
    // phases of each buffer in this launch (uniform over the cluster)
    const int n_phases =
        p.iters + ((p.sw_every > 0 && p.blur) ? p.iters / p.sw_every : 0) + (p.est ? 1 : 0);
    if (t == 0) {
        mbar_init(mb_r, 1);
        mbar_init(mb_c, 1);
        fence_mbar_init();
        mbar_arrive_expect(mb_r, G::PHASE_BYTES);
        mbar_arrive_expect(mb_c, G::PHASE_BYTES);
    }
    F::fill_twiddles(tw, p.tw, t, NT);
    auto pos = [&](int j, int s) { return q + TPL * j + R * s; };
    Cx<float> x[J][TPL];
    uint32_t in_bits = 0;  // bit TPL j + s: the support at (grow, pos(j, s))
    {
        const size_t pat = blockIdx.x / CL;
        const float* __restrict__ A = p.A + pat * p.a_stride;
        for (int i = t; i < L * RPC; i += NT) {
            const int f = i / RPC, c = i % RPC;
            Ac[c * ACP + f] = A[(size_t)f * L + rank * RPC + c];
        }
        const Cx<float>* __restrict__ X = p.x + pat * L * L + (size_t)grow * L;
        const float* __restrict__ S = p.S + pat * p.s_stride + (size_t)grow * L;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                x[j][s] = X[pos(j, s)];
                in_bits |= (S[pos(j, s)] > 0.5f ? 1u : 0u) << (TPL * j + s);
            }
    }
    auto inside = [&](int j, int s) { return (in_bits >> (TPL * j + s)) & 1u; };
    const bool neg = ((grow + q) & 1) != 0;
    auto sgn = [&](Cx<float> z) { return neg ? Cx<float>{-z.x, -z.y} : z; };

    bool ok = true;  // false once a wait ran out: no more waits or copies
    uint32_t par_r = 0, par_c = 0;
    int done_r = 0, done_c = 0;
    auto wait_phase = [&](uint32_t mb, uint32_t& par, int& done) {
        if (ok && !mbar_wait(mb, par, CLUSTER_WAIT_NS)) {
            ok = false;
            if (p.err) atomicExch(p.err, 1);
        }
        // the next phase of this buffer: no byte of it can have been sent yet
        if (t == 0 && ok && done + 1 < n_phases) mbar_arrive_expect(mb, G::PHASE_BYTES);
        par ^= 1u;
        ++done;
    };
    // forward row DFT of o into this row's slots; each CTA's block of columns to it
    auto rows_forward = [&](Cx<float>(&o)[J][TPL]) {
        Cx<float>* rw = rbuf + row * LS;
        Cx<float> v[R];
        F::template split_to_natural<false>(o, v, rw, 1, tw, q);
#pragma unroll
        for (int i = 0; i < R; ++i) rw[q + TPL * brev<R>(i)] = v[i];
        fence_proxy_async_smem();
        __syncwarp();
        // (failure test: the launch's first CTA withholds its first phase's
        // blocks, so its peers' waits for them run out)
        if (q < CL && ok && !(p.withhold && blockIdx.x == 0 && done_c == 0))
            bulk_copy_to_cta(cluster_map(cb + 8u * (uint32_t)(grow * CP), (uint32_t)q),
                             rb + 8u * (uint32_t)(row * LS + q * RPC), G::BLOCK_BYTES, cluster_map(mb_c, (uint32_t)q));
    };
    // column DFT, op per frequency, inverse column DFT of the arrived rows;
    // each CTA's block of rows to it
    auto columns = [&](auto op) {
        wait_phase(mb_c, par_c, done_c);
        Cx<float>* col = cbuf + cl;
        Cx<float> v[R];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = col[(qc + TPL * k) * CP];
        Cx<float> o[J][TPL];
        F::template natural_to_split<false>(v, o, col, CP, tw, qc);
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) o[j][s] = op(o[j][s], qc + TPL * j + R * s);
        F::template split_to_natural<true>(o, v, col, CP, tw, qc);
#pragma unroll
        for (int i = 0; i < R; ++i) col[(qc + TPL * brev<R>(i)) * CP] = v[i];
        fence_proxy_async_smem();
        __syncthreads();
        if (t < L && ok) {
            const int s = t / RPC, rl = t % RPC;  // global row t: local row rl of CTA s
            bulk_copy_to_cta(cluster_map(rb + 8u * (uint32_t)(rl * LS + rank * RPC), (uint32_t)s),
                             cb + 8u * (uint32_t)(t * CP), G::BLOCK_BYTES, cluster_map(mb_r, (uint32_t)s));
        }
    };
    // inverse row DFT of the arrived row into o
    auto rows_inverse = [&](Cx<float>(&o)[J][TPL]) {
        wait_phase(mb_r, par_r, done_r);
        Cx<float>* rw = rbuf + row * LS;
        Cx<float> v[R];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = rw[q + TPL * k];
        F::template natural_to_split<true>(v, o, rw, 1, tw, q);
    };
    auto modulus = [&](Cx<float> z, int f) { return data_apply(z, Ac[cl * ACP + f], DMODE); };
    __syncthreads();
    cluster_sync();  // every CTA running, its barriers initialised, before the first copy

    int update = 0;
    for (int it = 0; it < p.iters; ++it) {
        Cx<float> o[J][TPL];
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) o[j][s] = sgn(x[j][s]);
        rows_forward(o);
        columns(modulus);
        rows_inverse(o);
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                const Cx<float> y = sgn(cscale(o[j][s], p.scale));
                const bool keep = inside(j, s) && (!POS || y.x >= 0.0f);
                x[j][s] = keep ? y : merge_apply(y, x[j][s], -p.beta, 1.0f);
            }
        const bool update_next = p.sw_every > 0 && p.blur && (it + 1) % p.sw_every == 0;
        if (!update_next) continue;

        // ---- shrinkwrap: v = |x| blurred, support = { v > thresh * max v } ----
        for (int i = t; i < L; i += NT) gt[i] = p.blur[(size_t)update * L + i];
        ++update;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                const Cx<float> z = x[j][s];
                o[j][s] = sgn(Cx<float>{sqrtf(fmaf(z.x, z.x, z.y * z.y)), 0.0f});
            }
        rows_forward(o);
        // gt is read by the column phase after its wait, which follows the
        // __syncwarp and copies above; the block barrier makes it visible
        __syncthreads();
        columns([&](Cx<float> z, int f) { return cscale(z, gt[f] * gt[gcol]); });
        rows_inverse(o);
        float vmax = -INFINITY;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                o[j][s].x = sgn(cscale(o[j][s], p.scale)).x;
                vmax = fmaxf(vmax, o[j][s].x);
            }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
        if ((t & 31) == 0) red[warp] = vmax;
        __syncthreads();
        if (t < CL) {
            float m = red[0];
            for (int w = 1; w < G::WARPS; ++w) m = fmaxf(m, red[w]);
            cluster_store(cluster_map(cm + 4u * (uint32_t)rank, (uint32_t)t), m);
        }
        cluster_sync();
        float m = cmax[0];
#pragma unroll
        for (int r = 1; r < CL; ++r) m = fmaxf(m, cmax[r]);
        const float thr = p.thresh * m;
        in_bits = 0;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) in_bits |= (o[j][s].x > thr ? 1u : 0u) << (TPL * j + s);
    }
    {
        // x and the support out (addresses from the block index again)
        const size_t pat = cta_index() / CL;
        Cx<float>* __restrict__ Xo = p.x + pat * L * L + (size_t)grow * L;
        float* __restrict__ So = p.S + pat * p.s_stride + (size_t)grow * L;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) {
                Xo[pos(j, s)] = x[j][s];
                So[pos(j, s)] = inside(j, s) ? 1.0f : 0.0f;
            }
    }
    if (p.est) {
        // the estimate: the modulus projection of the final x, restricted to the support
        Cx<float> o[J][TPL];
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) o[j][s] = sgn(x[j][s]);
        rows_forward(o);
        columns(modulus);
        rows_inverse(o);
        Cx<float>* __restrict__ E = p.est + (cta_index() / CL) * L * L + (size_t)grow * L;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s)
                E[pos(j, s)] = inside(j, s) ? sgn(cscale(o[j][s], p.scale)) : Cx<float>{0.0f, 0.0f};
    }
    if (!ok) {
        // a wait ran out: give copies still in flight a bounded moment to land
        const uint64_t t0 = globaltimer_ns();
        while (globaltimer_ns() - t0 < 1000000ull) {
        }
    }
    // Every byte sent to this CTA has arrived (its last waits).  Once every
    // CTA is here no copy of the launch is in flight, and no CTA's shared
    // memory is read or written by another any more.
    cluster_sync();
}
template <int L, int CL>
cudaError_t hio_cluster_launch_cl(const HioDev& d, const HioArgs& a, cudaStream_t st) {
    using G = ClGeom<L, CL>;
    const bool always = (a.data_mode == DATA_ALWAYS);
    auto k = a.positivity ? (always ? k_hio_cl<L, CL, DATA_ALWAYS, true> : k_hio_cl<L, CL, DATA_SKIP_ZERO, true>)
                          : (always ? k_hio_cl<L, CL, DATA_ALWAYS, false> : k_hio_cl<L, CL, DATA_SKIP_ZERO, false>);
    const size_t smem = G::smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if constexpr (CL > 8) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(a.batch * CL));
    cfg.blockDim = dim3(G::NT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k, d);
    count_launches();
    return e != cudaSuccess ? e : cudaGetLastError();
}

HioDev hio_dev(const HioArgs& a, const void* tw) {
    HioDev d;
    d.x = (Cx<float>*)a.x;
    d.est = (Cx<float>*)a.estimate;
    d.A = (const float*)a.A;
    d.a_stride = a.a_stride;
    d.S = (float*)a.S;
    d.s_stride = a.s_stride;
    d.tw = (const Cx<float>*)tw;
    d.blur = (const float*)a.blur;
    d.err = a.err;
    d.withhold = a.withhold;
    d.scale = 1.0f / (float)(a.M * a.N);
    d.beta = (float)a.beta;
    d.thresh = (float)a.threshold;
    d.iters = a.iters;
    d.sw_every = a.sw_every;
    d.positivity = a.positivity;
    d.data_mode = a.data_mode;
    return d;
}

template <int L>
cudaError_t hio_launch(const HioArgs& a, const void* tw, cudaStream_t st) {
    const HioDev d = hio_dev(a, tw);
    const bool always = (a.data_mode == DATA_ALWAYS);
    if constexpr (L == 128) {
        if (a.tmem) {
            const size_t smem = hio_tm_smem_bytes();
            auto k = a.positivity ? (always ? k_hio_tm<DATA_ALWAYS, true> : k_hio_tm<DATA_SKIP_ZERO, true>)
                                  : (always ? k_hio_tm<DATA_ALWAYS, false> : k_hio_tm<DATA_SKIP_ZERO, false>);
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            k<<<(unsigned)a.batch, 1024, smem, st>>>(d);
            count_launches();
            return cudaGetLastError();
        }
    }
    const size_t smem = HioPlan<L>::smem_bytes();
    auto k = a.positivity ? (always ? k_hio<L, DATA_ALWAYS, true> : k_hio<L, DATA_SKIP_ZERO, true>)
                          : (always ? k_hio<L, DATA_ALWAYS, false> : k_hio<L, DATA_SKIP_ZERO, false>);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<(unsigned)a.batch, 4 * L, smem, st>>>(d);
    count_launches();
    return cudaGetLastError();
}

}  // namespace

bool hio_fused_supported(bool dbl, uint64_t M, uint64_t N) { return dm_fused_supported(dbl, M, N); }

bool hio_cluster_supported(bool dbl, uint64_t L, int cluster) {
    if (dbl) return false;
    if (L == 128) return cluster == 2 || cluster == 4 || cluster == 8;
    if (L == 256) return cluster == 8 || cluster == 16;
    return false;
}

size_t hio_cluster_smem_bytes(uint64_t L, int cluster) {
    if (L == 128) return cluster == 2 ? ClGeom<128, 2>::smem_bytes()
                         : cluster == 4 ? ClGeom<128, 4>::smem_bytes()
                                        : ClGeom<128, 8>::smem_bytes();
    return cluster == 8 ? ClGeom<256, 8>::smem_bytes() : ClGeom<256, 16>::smem_bytes();
}

namespace {
template <int L, int CL>
int hio_cluster_max_active_cl() {
    using G = ClGeom<L, CL>;
    auto k = k_hio_cl<L, CL, DATA_SKIP_ZERO, false>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes()) != cudaSuccess)
        return 0;
    if constexpr (CL > 8) {
        if (cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CL);
    cfg.blockDim = dim3(G::NT);
    cfg.dynamicSmemBytes = G::smem_bytes();
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return n;
}
}  // namespace

int hio_cluster_max_active(uint64_t L, int cluster) {
    if (!hio_cluster_supported(false, L, cluster)) return 0;
    if (L == 128) return cluster == 2 ? hio_cluster_max_active_cl<128, 2>()
                         : cluster == 4 ? hio_cluster_max_active_cl<128, 4>()
                                        : hio_cluster_max_active_cl<128, 8>();
    return cluster == 8 ? hio_cluster_max_active_cl<256, 8>() : hio_cluster_max_active_cl<256, 16>();
}

cudaError_t launch_hio_cluster(const HioArgs& a, int cluster, const void* tw, cudaStream_t st) {
    if (a.M != a.N || !hio_cluster_supported(false, a.M, cluster)) return cudaErrorInvalidValue;
    if (a.batch == 0 || (a.iters <= 0 && !a.estimate)) return cudaSuccess;
    const HioDev d = hio_dev(a, tw);
    if (a.M == 128) {
        switch (cluster) {
            case 2: return hio_cluster_launch_cl<128, 2>(d, a, st);
            case 4: return hio_cluster_launch_cl<128, 4>(d, a, st);
            case 8: return hio_cluster_launch_cl<128, 8>(d, a, st);
        }
    } else {
        switch (cluster) {
            case 8: return hio_cluster_launch_cl<256, 8>(d, a, st);
            case 16: return hio_cluster_launch_cl<256, 16>(d, a, st);
        }
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_hio_iterations(bool dbl, const HioArgs& a, const void* tw, cudaStream_t st) {
    if (!hio_fused_supported(dbl, a.M, a.N)) return cudaErrorInvalidValue;
    if (a.batch == 0 || (a.iters <= 0 && !a.estimate)) return cudaSuccess;
    switch (a.M) {
        case 32: return hio_launch<32>(a, tw, st);
        case 64: return hio_launch<64>(a, tw, st);
        case 128: return hio_launch<128>(a, tw, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cpra_b200
