// Line FFTs held in registers by small groups of cooperating threads.
//
// A line of power-of-two length L is split as L = R * TPL: each of TPL
// threads of one warp holds R = L / TPL values.  A forward transform is
//   X[m + R*s] = sum_q W_TPL^(q*s) * W_L^(q*m) * sum_k x[q + TPL*k] W_R^(k*m)
// i.e. an R-point DFT in registers, a twiddle by W_L^(q*m), one exchange of
// the line through shared memory, and a TPL-point DFT in registers.  The
// inverse runs the same steps in the opposite order.  Both directions are
// unnormalised; scaling is applied by the caller.
//
// Register layouts (q = the thread's rank in its group, 0 <= q < TPL):
//   natural : v[k]    = x[q + TPL*k]                  k < R
//   split   : o[j][s] = X[m_j + R*s],  m_j = q + TPL*j  j < R/TPL, s < TPL
// The caller loads and stores those positions; nothing is ever reordered in
// memory by a bit-reversal pass.
#pragma once
#include "cpra_common.cuh"

namespace cpra_b200 {

template <int R>
__host__ __device__ __forceinline__ constexpr int brev(int j) {
    int r = 0;
    for (int b = 1, t = R >> 1; b < R; b <<= 1, t >>= 1)
        if (j & b) r |= t;
    return r;
}

// a * W_32^k (forward: exp(-2 pi i k/32), inverse: exp(+2 pi i k/32)); k is a
// compile-time constant after unrolling, so the branches fold away and the
// multiplications by 1, -1, +-i are exact.
template <typename T, bool INV>
__device__ __forceinline__ Cx<T> rot32(Cx<T> a, int k) {
    k &= 31;
    if (k == 0) return a;
    if (k == 16) return cneg(a);
    if (k == 8) return INV ? Cx<T>{-a.y, a.x} : Cx<T>{a.y, -a.x};
    if (k == 24) return INV ? Cx<T>{a.y, -a.x} : Cx<T>{-a.y, a.x};
    const Cx<T> w = {tw32_cos<T>(k), INV ? tw32_sin<T>(k) : -tw32_sin<T>(k)};
    return cmul(a, w);
}

// In-place radix-2 decimation-in-frequency DFT of R <= 32 register values:
// natural order in, v[i] = X[brev<R>(i)] out.
template <typename T, int R, bool INV>
__device__ __forceinline__ void dft_regs(Cx<T> (&v)[R]) {
    static_assert(R >= 1 && R <= 32 && (R & (R - 1)) == 0, "R must be a power of two <= 32");
#pragma unroll
    for (int half = R / 2; half >= 1; half >>= 1) {
#pragma unroll
        for (int base = 0; base < R; base += 2 * half) {
#pragma unroll
            for (int j = 0; j < half; ++j) {
                const Cx<T> a = v[base + j];
                const Cx<T> b = v[base + j + half];
                v[base + j] = cadd(a, b);
                v[base + j + half] = rot32<T, INV>(csub(a, b), j * (32 / (2 * half)));
            }
        }
    }
}

// Exchange slot of element (m, q) in a line's L-slot scratch.  The rotation
// (q + m) mod TPL spreads both the writes (fixed m, all q) and the reads
// (fixed owned m_j and source p, all q) over distinct shared-memory banks for
// rows (slot stride 1, line stride L+TPL) and columns (slot stride L+TPL).
template <int TPL>
__device__ __forceinline__ int xslot(int m, int q) { return m * TPL + ((q + m) & (TPL - 1)); }

template <typename T, int L, int TPL>
struct LineFFT {
    static constexpr int R = L / TPL;
    // HALF: R = TPL / 2 (512 points over 32 threads, 16 values each); the
    // TPL-point second stage of each m is split over a lane pair by one
    // radix-2 step (natural_to_split_flat).  Otherwise TPL <= R.
    static constexpr bool HALF = (R < TPL);
    static constexpr int J = HALF ? 1 : R / TPL;
    static_assert(TPL >= 1 && TPL <= 32 && (TPL & (TPL - 1)) == 0, "TPL must be a power of two <= 32");
    static_assert(R <= 32 && (R >= TPL || (2 * R == TPL && TPL == 32)), "need TPL <= R <= 32, or R = TPL / 2 = 16");

    // Flat output layout of natural_to_split_flat: output i < R of rank q is
    // element pos(q, i) of the transformed line.  For TPL <= R this is the
    // split layout below, o[j][s] = flat[j * TPL + s]; for HALF, rank q holds
    // X[(q >> 1) + R (q & 1) + TPL i].
    __host__ __device__ __forceinline__ static constexpr int pos(int q, int i) {
        if constexpr (HALF)
            return (q >> 1) + R * (q & 1) + TPL * i;
        else
            return q + TPL * (i / TPL) + R * (i % TPL);
    }

    // Twiddle table layout: twq[p * TWS + m] = exp(-2 pi i p m / L) for p < TPL,
    // m < R.  The row pitch R + 1 puts the TPL ranks' entries for one m on
    // distinct shared-memory banks.
    static constexpr int TWS = R + 1;
    static constexpr int TW_ENTRIES = TPL * TWS;
    // fill a twiddle table from the full table tw[t] = exp(-2 pi i t / L)
    __device__ __forceinline__ static void fill_twiddles(Cx<T>* twq, const Cx<T>* __restrict__ tw, int tid,
                                                         int nthreads) {
        for (int i = tid; i < TW_ENTRIES; i += nthreads) {
            const int p = i / TWS, m = i % TWS;
            twq[i] = (m < R) ? tw[p * m] : Cx<T>{T(1), T(0)};
        }
    }

    // natural -> split.  scratch: the line's L slots in shared memory, slot u at
    // scratch[u * ss] (may be the storage the values were loaded from; the
    // group's warp is synchronised before it is overwritten); twq: the table
    // above.
    template <bool INV>
    __device__ __forceinline__ static void natural_to_split(Cx<T> (&v)[R], Cx<T> (&o)[J][TPL], Cx<T>* scratch,
                                                            int ss, const Cx<T>* twq, int q) {
        static_assert(!HALF || sizeof(T) == 0, "HALF lines use natural_to_split_flat");
        dft_regs<T, R, INV>(v);
        if constexpr (TPL == 1) {
#pragma unroll
            for (int j = 0; j < J; ++j) o[j][0] = v[brev<R>(j)];
        } else {
            __syncwarp();
#pragma unroll
            for (int m = 0; m < R; ++m) {
                Cx<T> y = v[brev<R>(m)];
                if (m != 0) y = INV ? cmulc(y, twq[q * TWS + m]) : cmul(y, twq[q * TWS + m]);
                scratch[xslot<TPL>(m, q) * ss] = y;
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int m = q + TPL * j;
                Cx<T> w[TPL];
#pragma unroll
                for (int p = 0; p < TPL; ++p) w[p] = scratch[xslot<TPL>(m, p) * ss];
                dft_regs<T, TPL, INV>(w);
#pragma unroll
                for (int s = 0; s < TPL; ++s) o[j][s] = w[brev<TPL>(s)];
            }
            __syncwarp();
        }
    }

    // natural -> flat (pos above).  For TPL <= R this is natural_to_split with
    // the outputs flattened.  For HALF: an R-point DFT over k of
    // x[q + TPL k], the twiddle W_L^(q m), the exchange, then for m = q >> 1
    // the TPL-point DFT over the ranks, X[m + R s] = sum_p W_TPL^(p s) Y_p[m],
    // as its even (q even) or odd (q odd) outputs: an R-point DFT of
    // Y_p + Y_(p+R), or of (Y_p - Y_(p+R)) W_TPL^p.
    template <bool INV>
    __device__ __forceinline__ static void natural_to_split_flat(Cx<T> (&v)[R], Cx<T> (&o)[R], Cx<T>* scratch,
                                                                 int ss, const Cx<T>* twq, int q) {
        if constexpr (!HALF) {
            natural_to_split<INV>(v, reinterpret_cast<Cx<T>(&)[J][TPL]>(o), scratch, ss, twq, q);
        } else {
            dft_regs<T, R, INV>(v);
            __syncwarp();
#pragma unroll
            for (int m = 0; m < R; ++m) {
                Cx<T> y = v[brev<R>(m)];
                if (m != 0) y = INV ? cmulc(y, twq[q * TWS + m]) : cmul(y, twq[q * TWS + m]);
                scratch[xslot<TPL>(m, q) * ss] = y;
            }
            __syncwarp();
            const int m = q >> 1;
            const bool odd = (q & 1) != 0;
            // a0 + sg * a1 as one fused multiply-add: the product by +-1 is
            // exact, so it rounds exactly like cadd (even) or csub (odd)
            const T sg = odd ? T(-1) : T(1);
            Cx<T> b[R];
#pragma unroll
            for (int p = 0; p < R; ++p) {
                const Cx<T> a0 = scratch[xslot<TPL>(m, p) * ss];
                const Cx<T> a1 = scratch[xslot<TPL>(m, p + R) * ss];
                const Cx<T> d = {fma_rn(sg, a1.x, a0.x), fma_rn(sg, a1.y, a0.y)};
                b[p] = odd ? rot32<T, INV>(d, p) : d;  // W_32^p (TPL = 32)
            }
            dft_regs<T, R, INV>(b);
#pragma unroll
            for (int i = 0; i < R; ++i) o[i] = b[brev<R>(i)];
            __syncwarp();
        }
    }

    // split -> natural (the reverse of natural_to_split's data movement)
    template <bool INV>
    __device__ __forceinline__ static void split_to_natural(Cx<T> (&o)[J][TPL], Cx<T> (&v)[R], Cx<T>* scratch,
                                                            int ss, const Cx<T>* twq, int q) {
        static_assert(!HALF || sizeof(T) == 0, "HALF lines have no split_to_natural");
        if constexpr (TPL == 1) {
#pragma unroll
            for (int m = 0; m < R; ++m) v[m] = o[m][0];
        } else {
            __syncwarp();
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int m = q + TPL * j;
                Cx<T> w[TPL];
#pragma unroll
                for (int s = 0; s < TPL; ++s) w[s] = o[j][s];
                dft_regs<T, TPL, INV>(w);  // w[i] = Z[m][brev(i)]
#pragma unroll
                for (int i = 0; i < TPL; ++i) {
                    const int p = brev<TPL>(i);
                    Cx<T> z = w[i];
                    if (p * m != 0) z = INV ? cmulc(z, twq[p * TWS + m]) : cmul(z, twq[p * TWS + m]);
                    scratch[xslot<TPL>(m, p) * ss] = z;
                }
            }
            __syncwarp();
#pragma unroll
            for (int m = 0; m < R; ++m) v[m] = scratch[xslot<TPL>(m, q) * ss];
            __syncwarp();
        }
        dft_regs<T, R, INV>(v);  // v[i] = x[q + TPL * brev<R>(i)]
    }
};

}  // namespace cpra_b200
