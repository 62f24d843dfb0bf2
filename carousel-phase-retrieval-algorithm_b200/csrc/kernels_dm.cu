// Fused difference-map iterations: the reference's 12-call iteration
// (src/CPRA_MKL.cpp:94-110)
//   t1 <- Forward2D; DataConstraint(A); Backward2D; t1 <- a1*x + b1*t1; SpaceConstraint(S)
//   t2 <- SpaceConstraint(S); t2 <- a2*x + b2*t2; Forward2D; DataConstraint(A); Backward2D
//   x  <- a3*t1 + b3*x;  x <- a4*t2 + b4*x
// as one kernel with one CTA per pattern and `iters` iterations per launch.
//
// On chip for the whole launch: the plane buffer of the transforms, the
// modulus plane A and the support (as a bit mask) in shared memory, and t1 --
// real after SpaceConstraint -- in registers: every row thread reads and
// writes its row in the same split positions (fft2d_cta.cuh), so the value a
// thread produces for t1 is the value it consumes next.  Only x and t2 travel
// through global memory (L2): the second half of each iteration already forms
// the next iteration's a2*x + b2*S(t2), so each iteration reads that one
// plane and x, and writes x and t2 once.  The first half's update needs x a
// second time; half of those values come from registers (the new x the
// previous iteration left there, carried through the transforms in t1's
// registers, which are free in that half), the other half from L2, loaded
// together with the second half's t2.  The fftshifts cancel in pairs
// around the modulus step (DataConstraint commutes with the (-1)^(i+j) sign
// pattern), leaving sign flips on the input of each forward and the output of
// each inverse transform.
//
// The arithmetic is the per-operator kernels' arithmetic step for step
// (Plane<> passes, ops_ew.cuh operators), so one launch with `iters`
// iterations writes the same bits as 12*iters per-operator calls.
#include "cpra_internal.h"
#include "fft2d_cta.cuh"
#include "ops_ew.cuh"
#include "tmem.cuh"

namespace cpra_b200 {

namespace {

struct DmDev {
    Cx<float>* x;
    Cx<float>* t1;
    Cx<float>* t2;
    const Cx<float>* xprev;
    const Cx<float>* xnext;
    int mix, init_from_x;
    const float* A;
    uint64_t a_stride;
    const float* S;
    uint64_t s_stride;
    const Cx<float>* tw;
    float scale;
    float a1, b1, a2, b2, a3, b3, a4, b4;
    int iters, space_mode, data_mode;
};

// The plane of the fused kernel: the same thread split as the per-operator
// transforms of this size (plane_tpl), so both round identically.
template <int L>
using DmP = Plane<float, L, plane_tpl<float, L>()>;

// Shared memory of one CTA: the plane buffer, A with row pitch AP, the
// twiddle table, and the support as a bit mask (SpaceConstraint's threshold
// test evaluated once per launch: bit set where the value is kept), MP words
// per row.  The column pass reads A[f][c] for the TPL ranks' rows f and the
// warp's 32 / TPL columns c: AP = L + 8 (4 ranks x 8 columns) or L + 4
// (8 ranks x 4 columns) puts them on distinct banks.  With 8 threads per line
// a row pass's warp takes rows 4 apart, and a mask row pitch of L/32 + 1
// words keeps their mask words on distinct banks.
template <int L>
struct DmPlan {
    using P = DmP<L>;
    static constexpr int AP = (P::TPL == 8) ? L + 4 : L + 8;
    static constexpr int MP = L / 32 + ((P::TPL == 8) ? 1 : 0);
    static constexpr int MASK_WORDS = L * MP;
    static constexpr size_t a_bytes() { return sizeof(float) * (size_t)L * AP; }
    static constexpr size_t smem_bytes() {
        return P::buf_bytes() + a_bytes() + P::tw_bytes() + sizeof(uint32_t) * MASK_WORDS;
    }
    __device__ __forceinline__ static bool mask_keep(const uint32_t* mask, int idx) {
        return (mask[(idx / L) * MP + (idx % L) / 32] >> (idx & 31)) & 1u;
    }
    // the CTA's threads fill the mask from the support plane S
    __device__ __forceinline__ static void fill_mask(uint32_t* mask, const float* __restrict__ S, int t) {
        for (int i = t; i < L * L; i += P::NT) {
            const unsigned keep = __ballot_sync(0xffffffffu, !space_zero(S[i]));
            if ((i & 31) == 0) mask[(i / L) * MP + (i % L) / 32] = keep;
        }
    }
};

// column forward transform, modulus projection (DataConstraint mode DMODE),
// column inverse transform
template <int L, int DMODE>
__device__ __forceinline__ void modulus_columns(Cx<float>* buf, const Cx<float>* tw, const float* As, int c, int q) {
    using P = DmP<L>;
    constexpr int AP = DmPlan<L>::AP;
    Cx<float> o[P::J][P::TPL];
    P::template col_from_buf<false>(o, buf, tw, c, q);
#pragma unroll
    for (int j = 0; j < P::J; ++j)
#pragma unroll
        for (int s = 0; s < P::TPL; ++s) {
            const int f = P::split_pos(q, j, s);
            o[j][s] = data_apply(o[j][s], As[f * AP + c], DMODE);
        }
    P::template col_to_buf<true>(o, buf, tw, c, q);
}

// SMODE / DMODE: the SpaceConstraint and DataConstraint modes, fixed at
// compile time so that each instantiation carries only its own arithmetic.
// At 64^2 two CTAs share an SM (at most 128 registers, no spills; left
// unbounded the kernel takes 155 and one CTA per SM).
template <int L, int SMODE, int DMODE>
__global__ void __launch_bounds__(DmP<L>::NT, (L == 64) ? 2 : 1) k_dm(const DmDev p) {
    using P = DmP<L>;
    using D = DmPlan<L>;
    constexpr int J = P::J, TPL = P::TPL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* buf = reinterpret_cast<Cx<float>*>(smem_raw);
    float* As = reinterpret_cast<float*>(smem_raw + P::buf_bytes());
    Cx<float>* tw = reinterpret_cast<Cx<float>*>(smem_raw + P::buf_bytes() + D::a_bytes());
    uint32_t* mask = reinterpret_cast<uint32_t*>(smem_raw + P::buf_bytes() + D::a_bytes() + P::tw_bytes());
    const int t = threadIdx.x, line = P::row_of(t), col = P::col_of(t), q = P::rank_of(t);
    P::F::fill_twiddles(tw, p.tw, t, P::NT);
    const size_t base = (size_t)blockIdx.x * L * L;
    Cx<float>* __restrict__ X = p.x + base;
    Cx<float>* __restrict__ T1 = p.t1 + base;
    Cx<float>* __restrict__ T2 = p.t2 + base;
    const Cx<float>* __restrict__ XP = p.xprev + (p.xprev ? base : 0);
    const Cx<float>* __restrict__ XN = p.xnext + (p.xnext ? base : 0);
    const float* __restrict__ A = p.A + blockIdx.x * p.a_stride;
    const float* __restrict__ S = p.S + blockIdx.x * p.s_stride;
    for (int i = t; i < L * L; i += P::NT) As[(i / L) * D::AP + (i % L)] = A[i];
    constexpr bool use_mask = (SMODE == SPACE_THRESHOLD);
    if constexpr (use_mask) D::fill_mask(mask, S, t);
    // SpaceConstraint of element idx, from the mask or the support plane
    auto space = [&](Cx<float> z, int idx) -> Cx<float> {
        if constexpr (use_mask)
            return {D::mask_keep(mask, idx) ? z.x : 0.0f, 0.0f};
        else
            return space_apply(z, S[idx], SMODE);
    };
    // every element this thread touches has index line*L + split_pos(q, j, s)
    auto at = [&](int j, int s) { return line * L + P::split_pos(q, j, s); };
    // (-1)^(row + col) is the same for all of them
    const bool neg = ((line + q) & 1) != 0;
    auto sgn = [&](Cx<float> z) { return neg ? Cx<float>{-z.x, -z.y} : z; };
    float t1r[J][TPL];
    __syncthreads();

    // Both halves of an iteration run through one loop body, so each transform
    // pass exists once in the binary (the fully unrolled passes are large and
    // duplicating them overflows the instruction cache).  Between halves no
    // block barrier is needed: a row's slots in the plane buffer are only
    // touched by the four threads of that row, which share a warp.
    Cx<float> o[J][TPL];
    for (int it = 0; it < p.iters; ++it) {
        const bool last = (it == p.iters - 1);
#pragma unroll 1
        for (int ph = 0; ph < 2; ++ph) {
            if (ph == 0) {
                // t1 <- S( a1*x + b1*Backward2D(DataConstraint(Forward2D(t1))) )
                if (it > 0) {
                    // o[j < J/2] holds the previous iteration's new x there
                    // (second half's last step); t1's registers take it over
#pragma unroll
                    for (int j = 0; j < J / 2; ++j)
#pragma unroll
                        for (int s = 0; s < TPL; ++s) {
                            const Cx<float> xv = o[j][s];
                            o[j][s] = sgn(Cx<float>{t1r[j][s], 0.0f});
                            o[j + J / 2][s] = sgn(Cx<float>{t1r[j + J / 2][s], 0.0f});
                            t1r[j][s] = xv.x;
                            t1r[j + J / 2][s] = xv.y;
                        }
                } else if (!p.init_from_x) {
#pragma unroll
                    for (int j = 0; j < J; ++j)
#pragma unroll
                        for (int s = 0; s < TPL; ++s) o[j][s] = sgn(T1[at(j, s)]);
                } else {
                    // the angle's start: carousel mix of x, then t1 = t2 = x (:64-80)
#pragma unroll
                    for (int j = 0; j < J; ++j)
#pragma unroll
                        for (int s = 0; s < TPL; ++s) {
                            const int idx = at(j, s);
                            Cx<float> xv = X[idx];
                            if (p.mix == MIX_FIRST) {
                                xv = merge_apply(XN[idx], xv, 0.5f, 0.5f);
                            } else if (p.mix == MIX_LAST) {
                                xv = merge_apply(XP[idx], xv, 0.5f, 0.5f);
                            } else if (p.mix == MIX_MIDDLE) {
                                xv = merge_apply(XP[idx], xv, 0.5f, 0.0f);
                                xv = merge_apply(XN[idx], xv, 0.5f, 1.0f);
                            }
                            if (p.mix != MIX_NONE) X[idx] = xv;
                            o[j][s] = sgn(xv);
                        }
                }
                // t1's registers are free until this half's last step: they
                // carry the first J/2 split columns of this row's x (real
                // parts in t1r[j], imaginary parts in t1r[j + J/2]); on the
                // first iteration they are loaded now, so that the transforms
                // hide the latency
                if (it == 0) {
#pragma unroll
                    for (int j = 0; j < J / 2; ++j)
#pragma unroll
                        for (int s = 0; s < TPL; ++s) {
                            const Cx<float> xv = X[at(j, s)];
                            t1r[j][s] = xv.x;
                            t1r[j + J / 2][s] = xv.y;
                        }
                }
            } else {
                // t2 <- Backward2D(DataConstraint(Forward2D( a2*x + b2*S(t2) )))
                // (from the second iteration on, T2 already holds a2*x + b2*S(t2);
                // on an angle's start t2 = x)
#pragma unroll
                for (int j = 0; j < J; ++j)
#pragma unroll
                    for (int s = 0; s < TPL; ++s) {
                        const int idx = at(j, s);
                        Cx<float> z;
                        if (it > 0) {
                            z = o[j][s];  // loaded by the first half's last step
                        } else {
                            const Cx<float> xv = X[idx];
                            z = merge_apply(xv, space(p.init_from_x ? xv : T2[idx], idx), p.a2, p.b2);
                        }
                        o[j][s] = (it > 0) ? z : sgn(z);
                    }
            }
            P::template rows_split_to_buf<false>(o, buf, tw, line, q);
            __syncthreads();
            modulus_columns<L, DMODE>(buf, tw, As, col, q);
            __syncthreads();
            P::template row_from_buf<true>(o, buf, tw, line, q);
            if (ph == 0) {
#pragma unroll
                for (int j = 0; j < J; ++j)
#pragma unroll
                    for (int s = 0; s < TPL; ++s) {
                        const Cx<float> val = sgn(cscale(o[j][s], p.scale));
                        // j < J/2: x from t1's registers (read before t1r[j] is
                        // overwritten; t1r[j + J/2] is overwritten later)
                        const Cx<float> xv = (j < J / 2) ? Cx<float>{t1r[j][s], t1r[j + J / 2][s]} : X[at(j, s)];
                        const Cx<float> m = space(merge_apply(xv, val, p.a1, p.b1), at(j, s));
                        t1r[j][s] = m.x;
                        if (last) T1[at(j, s)] = m;
                        if (it > 0) o[j][s] = sgn(T2[at(j, s)]);
                    }
            } else {
#pragma unroll
                for (int j = 0; j < J; ++j)
#pragma unroll
                    for (int s = 0; s < TPL; ++s) {
                        const int idx = at(j, s);
                        const Cx<float> t2n = sgn(cscale(o[j][s], p.scale));
                        const Cx<float> x1 = merge_apply(Cx<float>{t1r[j][s], 0.0f}, X[idx], p.a3, p.b3);
                        const Cx<float> xn = merge_apply(t2n, x1, p.a4, p.b4);
                        X[idx] = xn;
                        T2[idx] = last ? t2n : merge_apply(xn, space(t2n, idx), p.a2, p.b2);
                        if (j < J / 2) o[j][s] = xn;  // for the next iteration's first half
                    }
            }
        }
    }
}

// The 128 x 128 kernel with its iterates resident in tensor memory.
//
// Every thread reads and writes x, t1 and t2 only at its own row's split
// positions (row*L + split_pos(q, j, s)), so these planes are thread-private
// for the whole launch.  They live in the SM's 256 KB of tensor memory, which
// holds one pattern's x and t2 (2 x 128 KB) exactly; t1, real after the
// support projection, takes t2's place between the first half's last step
// (which reads t2) and the second half's last step (which writes it).  So a
// thread's registers hold only the 16 values of its line segment, and the
// CTA runs 1024 threads (8 per line, 32 warps per SM) where k_dm runs 512.
// Warp w's threads own lane 32*(w % 4) + lane id, columns (w / 4)*64 .. +63:
// x at 0..31 (element (j, s) at 2*(8j + s), re then im), t2 or t1 at 32..63.
// Global memory is read when the launch starts (x with the carousel mix, t1
// and t2, or t1 = t2 = x) and written after the last iteration (x, t1, t2),
// so a launch of `iters` iterations moves each plane through L2/HBM once
// instead of once per iteration.  The arithmetic is k_dm's, step for step:
// both write the same bits.
//
// 512 columns are allocated per CTA; the 199 KB of shared memory allow one
// CTA per SM, so the allocation never waits for another CTA.
template <int SMODE, int DMODE>
__global__ void __launch_bounds__(1024, 1) k_dm_tm(const DmDev p) {
    constexpr int L = 128;
    using P = DmP<L>;
    using D = DmPlan<L>;
    constexpr int J = P::J, TPL = P::TPL;
    static_assert(TPL == 8 && J == 2 && P::NT == 1024, "two 8-value groups per thread, 32 warps");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t tm_base;
    Cx<float>* buf = reinterpret_cast<Cx<float>*>(smem_raw);
    float* As = reinterpret_cast<float*>(smem_raw + P::buf_bytes());
    Cx<float>* tw = reinterpret_cast<Cx<float>*>(smem_raw + P::buf_bytes() + D::a_bytes());
    const int t = threadIdx.x, row = P::row_of(t), col = P::col_of(t), q = P::rank_of(t), warp = t >> 5;
    if (warp == 0) tm_alloc(&tm_base, 512);
    P::F::fill_twiddles(tw, p.tw, t, P::NT);
    const size_t base = (size_t)blockIdx.x * L * L;
    Cx<float>* __restrict__ X = p.x + base;
    Cx<float>* __restrict__ T1 = p.t1 + base;
    Cx<float>* __restrict__ T2 = p.t2 + base;
    const Cx<float>* __restrict__ XP = p.xprev + (p.xprev ? base : 0);
    const Cx<float>* __restrict__ XN = p.xnext + (p.xnext ? base : 0);
    const float* __restrict__ A = p.A + blockIdx.x * p.a_stride;
    const float* __restrict__ S = p.S + blockIdx.x * p.s_stride;
    for (int i = t; i < L * L; i += P::NT) As[(i / L) * D::AP + (i % L)] = A[i];
    constexpr bool use_mask = (SMODE == SPACE_THRESHOLD);
    auto at = [&](int j, int s) { return row * L + P::split_pos(q, j, s); };
    // the threshold SpaceConstraint of this thread's 16 pixels, evaluated once
    // per launch: bit 8j + s set where the value is kept
    uint32_t keep_bits = 0;
    if constexpr (use_mask) {
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int s = 0; s < TPL; ++s) keep_bits |= (space_zero(S[at(j, s)]) ? 0u : 1u) << (TPL * j + s);
    }
    // SpaceConstraint of element (j, s) of this thread
    auto space = [&](Cx<float> z, int j, int s) -> Cx<float> {
        if constexpr (use_mask)
            return {((keep_bits >> (TPL * j + s)) & 1u) ? z.x : 0.0f, 0.0f};
        else
            return space_apply(z, S[at(j, s)], SMODE);
    };
    const bool neg = ((row + q) & 1) != 0;
    auto sgn = [&](Cx<float> z) { return neg ? Cx<float>{-z.x, -z.y} : z; };
    tm_fence_before_sync();
    __syncthreads();
    tm_fence_after_sync();
    // this thread's strip; the values of (j, s) with s in [4h, 4h + 4) are
    // group g = 2j + h: x at xa + 8g, t2 (or t1, 4 columns) at ta + 8g
    const uint32_t xa = tm_lane_addr(tm_base, warp, (warp >> 2) * 64);
    const uint32_t ta = xa + 32;
    Cx<float> o[J][TPL];
    // the launch's start: x (after the carousel mix) and t2 into tensor
    // memory, the first half's input t1 into o
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            Cx<float> xs[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int idx = at(j, 4 * h + u);
                Cx<float> xv = X[idx];
                if (!p.init_from_x) {
                } else if (p.mix == MIX_FIRST) {
                    xv = merge_apply(XN[idx], xv, 0.5f, 0.5f);
                } else if (p.mix == MIX_LAST) {
                    xv = merge_apply(XP[idx], xv, 0.5f, 0.5f);
                } else if (p.mix == MIX_MIDDLE) {
                    xv = merge_apply(XP[idx], xv, 0.5f, 0.0f);
                    xv = merge_apply(XN[idx], xv, 0.5f, 1.0f);
                }
                xs[u] = xv;
            }
            tm_st4(xa + 8 * (2 * j + h), xs);
            if (p.init_from_x) {
#pragma unroll
                for (int u = 0; u < 4; ++u) o[j][4 * h + u] = sgn(xs[u]);
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int idx = at(j, 4 * h + u);
                    o[j][4 * h + u] = sgn(T1[idx]);
                    xs[u] = T2[idx];
                }
                tm_st4(ta + 8 * (2 * j + h), xs);
            }
        }
    for (int it = 0; it < p.iters; ++it) {
        const bool last = (it == p.iters - 1);
        // the two halves unrolled: each transform pass is half of k_dm's code
        // (16 values per thread), so both copies fit the instruction cache
#pragma unroll
        for (int ph = 0; ph < 2; ++ph) {
            // first half:  t1' = Backward2D(DataConstraint(Forward2D(t1)))
            // second half: t2' = Backward2D(DataConstraint(Forward2D(a2*x + b2*S(t2))))
            P::template rows_split_to_buf<false>(o, buf, tw, row, q);
            __syncthreads();
            modulus_columns<L, DMODE>(buf, tw, As, col, q);
            __syncthreads();
            P::template row_from_buf<true>(o, buf, tw, row, q);
            if (ph == 0) {
                // t1 <- S(a1*x + b1*t1') into t2's columns once t2 is read;
                // o takes the second half's input
#pragma unroll
                for (int j = 0; j < J; ++j)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int g = 2 * j + h;
                        Cx<float> xr[4], tv[4];
                        float t1v[4];
                        tm_ld4(xa + 8 * g, xr);
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int s = 4 * h + u;
                            const Cx<float> val = sgn(cscale(o[j][s], p.scale));
                            t1v[u] = space(merge_apply(xr[u], val, p.a1, p.b1), j, s).x;
                        }
                        if (it > 0) {
                            // a2*x + b2*S(t2), formed by the previous iteration
                            tm_ld4(ta + 8 * g, tv);
#pragma unroll
                            for (int u = 0; u < 4; ++u) o[j][4 * h + u] = sgn(tv[u]);
                        } else {
                            // t2 from the buffer, or t2 = x on an angle's start
                            if (p.init_from_x) {
#pragma unroll
                                for (int u = 0; u < 4; ++u) tv[u] = xr[u];
                            } else {
                                tm_ld4(ta + 8 * g, tv);
                            }
#pragma unroll
                            for (int u = 0; u < 4; ++u)
                                o[j][4 * h + u] =
                                    sgn(merge_apply(xr[u], space(tv[u], j, 4 * h + u), p.a2, p.b2));
                        }
                        tm_st4r(ta + 8 * g, t1v);
                    }
            } else {
                // x <- a3*t1 + b3*x; x <- a4*t2' + b4*x; t2's columns take the
                // next iteration's a2*x + b2*S(t2') (after the last iteration
                // t2' itself); o takes the next first half's input t1
#pragma unroll
                for (int j = 0; j < J; ++j)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int g = 2 * j + h;
                        Cx<float> xr[4], tn[4];
                        float t1v[4];
                        tm_ld4_4r(xa + 8 * g, ta + 8 * g, xr, t1v);
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int s = 4 * h + u;
                            const Cx<float> t2n = sgn(cscale(o[j][s], p.scale));
                            const Cx<float> x1 = merge_apply(Cx<float>{t1v[u], 0.0f}, xr[u], p.a3, p.b3);
                            const Cx<float> xn = merge_apply(t2n, x1, p.a4, p.b4);
                            xr[u] = xn;
                            tn[u] = last ? t2n : merge_apply(xn, space(t2n, j, s), p.a2, p.b2);
                            o[j][s] = sgn(Cx<float>{t1v[u], 0.0f});
                        }
                        tm_st4(xa + 8 * g, xr);
                        tm_st4(ta + 8 * g, tn);
                    }
            }
        }
    }
    // write-out: x and t2 from tensor memory, t1 (= SpaceConstraint's
    // {value, 0}) from the first half's input in o
    if (p.iters > 0) {
        // the plane's addresses again from the block index (read anew, so that
        // no pointer stays in a register through the iterations)
        const size_t b2 = (size_t)cta_index() * L * L;
        Cx<float>* __restrict__ Xo = p.x + b2;
        Cx<float>* __restrict__ T1o = p.t1 + b2;
        Cx<float>* __restrict__ T2o = p.t2 + b2;
#pragma unroll
        for (int j = 0; j < J; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int g = 2 * j + h;
                Cx<float> xr[4], tv[4];
                tm_ld4(xa + 8 * g, xr);
                tm_ld4(ta + 8 * g, tv);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int idx = at(j, 4 * h + u);
                    Xo[idx] = xr[u];
                    T2o[idx] = tv[u];
                    T1o[idx] = sgn(o[j][4 * h + u]);
                }
            }
    }
    tm_wait_st();
    tm_fence_before_sync();
    __syncthreads();
    tm_fence_after_sync();
    if (warp == 0) tm_free(tm_base, 512);
}

template <int L>
cudaError_t dm_launch(const DmArgs& a, const void* tw, cudaStream_t st) {
    DmDev d;
    d.x = (Cx<float>*)a.x;
    d.t1 = (Cx<float>*)a.t1;
    d.t2 = (Cx<float>*)a.t2;
    d.xprev = (const Cx<float>*)a.xprev;
    d.xnext = (const Cx<float>*)a.xnext;
    d.mix = a.mix;
    d.init_from_x = a.init_from_x;
    d.A = (const float*)a.A;
    d.a_stride = a.a_stride;
    d.S = (const float*)a.S;
    d.s_stride = a.s_stride;
    d.tw = (const Cx<float>*)tw;
    d.scale = 1.0f / (float)(a.M * a.N);  // DFTI_BACKWARD_SCALE (include/MKL_Impl.hpp:40)
    d.a1 = (float)a.c.a1;
    d.b1 = (float)a.c.b1;
    d.a2 = (float)a.c.a2;
    d.b2 = (float)a.c.b2;
    d.a3 = (float)a.c.a3;
    d.b3 = (float)a.c.b3;
    d.a4 = (float)a.c.a4;
    d.b4 = (float)a.c.b4;
    d.iters = a.iters;
    d.space_mode = a.space_mode;
    d.data_mode = a.data_mode;
    const size_t smem = DmPlan<L>::smem_bytes();
    auto k = (a.space_mode == SPACE_THRESHOLD)
                 ? (a.data_mode == DATA_ALWAYS ? k_dm<L, SPACE_THRESHOLD, DATA_ALWAYS>
                                               : k_dm<L, SPACE_THRESHOLD, DATA_SKIP_ZERO>)
                 : (a.data_mode == DATA_ALWAYS ? k_dm<L, SPACE_POSITIVE_SCALED, DATA_ALWAYS>
                                               : k_dm<L, SPACE_POSITIVE_SCALED, DATA_SKIP_ZERO>);
    if constexpr (L == 128) {
        if (a.tmem)
            k = (a.space_mode == SPACE_THRESHOLD)
                    ? (a.data_mode == DATA_ALWAYS ? k_dm_tm<SPACE_THRESHOLD, DATA_ALWAYS>
                                                  : k_dm_tm<SPACE_THRESHOLD, DATA_SKIP_ZERO>)
                    : (a.data_mode == DATA_ALWAYS ? k_dm_tm<SPACE_POSITIVE_SCALED, DATA_ALWAYS>
                                                  : k_dm_tm<SPACE_POSITIVE_SCALED, DATA_SKIP_ZERO>);
    }
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<(unsigned)a.batch, DmP<L>::NT, smem, st>>>(d);
    count_launches();
    return cudaGetLastError();
}

template <int L>
int dm_occupancy() {
    const size_t smem = DmPlan<L>::smem_bytes();
    auto k = k_dm<L, SPACE_THRESHOLD, DATA_SKIP_ZERO>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 1;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, DmP<L>::NT, smem) != cudaSuccess || n < 1) return 1;
    return n;
}

}  // namespace

int dm_fused_ctas_per_sm(uint64_t M) {
    switch (M) {
        case 32: return dm_occupancy<32>();
        case 64: return dm_occupancy<64>();
        case 128: return dm_occupancy<128>();
        default: return 1;
    }
}

bool dm_fused_supported(bool dbl, uint64_t M, uint64_t N) {
    return !dbl && M == N && (M == 32 || M == 64 || M == 128);
}

cudaError_t launch_dm_iterations(bool dbl, const DmArgs& a, const void* tw, cudaStream_t st) {
    if (!dm_fused_supported(dbl, a.M, a.N)) return cudaErrorInvalidValue;
    if (a.batch == 0 || a.iters <= 0) return cudaSuccess;
    switch (a.M) {
        case 32: return dm_launch<32>(a, tw, st);
        case 64: return dm_launch<64>(a, tw, st);
        case 128: return dm_launch<128>(a, tw, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cpra_b200
