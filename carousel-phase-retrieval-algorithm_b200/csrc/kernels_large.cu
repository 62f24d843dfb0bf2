// HIO with shrinkwrap support updates for planes too large for one CTA
// (256 x 256 and 512 x 512, float): the same iteration as the one-CTA kernel
// (kernels_hio.cu; project-defined algorithm) as line passes, each moving the
// plane through L2 once:
//   columns  Y <- column IDFT(op(column DFT(Y)))                    k_big_cols
//            op = the modulus projection with A, or the Gaussian blur
//            transfer g(f_row) g(f_col) of a shrinkwrap update
//   rows     y = D (.) row IDFT(Y) / (MN), then                      k_big_rows
//            the HIO update of x with the support followed by the next
//            iteration's forward row transform Y <- row DFT(D (.) x), or the
//            blurred |x| and its per-pattern maximum, or the estimate S (.) y
// so an iteration is two passes (Y <- row DFT(D (.) x) before the first:
// k_big_rows_fwd, which after a shrinkwrap blur also writes the new support)
// with D = (-1)^(row + col) folding the fftshifts (the centred transform of
// an even-sized plane is D (.) DFT(D (.) x); the modulus step commutes with
// D).  Patterns run in chunks (all of them by default: a chunk sized to stay
// in L2 measured slower on B200 than whole-batch passes, whose larger grids
// keep every SM busy), each chunk through all iterations.
//
// Lines follow line_pass.cuh's LineGeom (16 values per thread; 16 threads per
// line at 256, 32 at 512).  Transforms take their line in natural order
// (LineFFT::natural_to_split_flat) and leave it in the flat layout.  Where a
// second transform follows, at 256 it runs straight from the split layout in
// registers (split_to_natural); at 512 (no such inverse for the half-split
// form) the values go back through the line's shared slots.  Row passes stage Y and x tiles with cp.async and write global
// memory directly (a thread group's outputs for one i are consecutive
// elements); the column pass stages a tile of columns of Y and A.  Per
// iteration the passes move 52 bytes and a bit per pixel (rows: Y, x read and
// written, the support mask; columns: Y read and written, A read).
#include "cpra_internal.h"
#include "line_pass.cuh"
#include "ops_ew.cuh"

namespace cpra_b200 {
namespace {

template <int L>
struct Big : LineGeom<L> {
    using G = LineGeom<L>;
    using F = typename G::F;
    static constexpr int TPL = G::TPL, R = G::R, NT = G::THREADS;
    static constexpr int RL = G::ROW_LINES, CL = G::COL_LINES, CS = G::CS, AS = G::AS;
    static constexpr size_t tile = G::row_tile;
    static constexpr int MW = L / 32;  // support mask words per row
    // CTAs per SM the register budget is sized for (80 registers; shared
    // memory allows 3 as well)
    static constexpr int MINB = 3;
    // rows: Y tile (also the exchange scratch), x tile, twiddles, mask tile, max
    static constexpr size_t row_smem() { return sizeof(Cx<float>) * (2 * tile + F::TW_ENTRIES) + tile / 8 + 16; }
    static constexpr size_t col_smem() {
        return sizeof(Cx<float>) * ((size_t)L * CS + F::TW_ENTRIES) + sizeof(float) * ((size_t)L * AS + L);
    }
};

// Y's row from the line's natural-order values v (already D-flipped): the
// forward transform (scratch: the line's shared slots), stored in the flat layout
template <int L>
__device__ __forceinline__ void big_row_forward(Cx<float> (&v)[Big<L>::R], Cx<float>* scratch, const Cx<float>* tw,
                                                int q, Cx<float>* __restrict__ yr) {
    using B = Big<L>;
    Cx<float> o[B::R];
    B::F::template natural_to_split_flat<false>(v, o, scratch, 1, tw, q);
#pragma unroll
    for (int i = 0; i < B::R; ++i) yr[B::pos(q, i)] = o[i];
}

// Y <- row DFT of D (.) x; with V: also the support mask <- { V > threshold *
// vmax } (the support of a shrinkwrap update).  vec_x: x rows 16-byte aligned
template <int L>
__global__ void __launch_bounds__(Big<L>::NT, Big<L>::MINB) k_big_rows_fwd(const Cx<float>* __restrict__ x,
                                                                Cx<float>* __restrict__ Y,
                                                                const Cx<float>* __restrict__ twg,
                                                                const float* __restrict__ V,
                                                                const unsigned int* __restrict__ vmax,
                                                                uint32_t* __restrict__ mask, float threshold,
                                                                int vec_x) {
    using B = Big<L>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* Yt = reinterpret_cast<Cx<float>*>(smem_raw);
    Cx<float>* Xt = Yt + B::tile;
    Cx<float>* tw = Xt + B::tile;
    int line, q;
    B::row_lane(threadIdx.x, line, q);
    const int t = threadIdx.x;
    const uint64_t g0 = (uint64_t)blockIdx.x * B::RL;  // first row of the chunk's [batch*L][L] plane stack
    stage(Xt, x + g0 * L, (uint32_t)(B::tile * 8), vec_x, t, B::NT);
    cp_async_commit();
    B::F::fill_twiddles(tw, twg, t, B::NT);
    const uint64_t g = g0 + line, b = g / L;
    const int r = (int)(g % L);
    if (V) {
        // lanes of a row hold TPL consecutive pixels TPL k + q: a 32-thread
        // line fills one mask word per k, a 16-thread line half of one (the
        // warp's other half is the next row)
        const float thr = threshold * unordered(vmax[b]);
        const float* __restrict__ Vr = V + g * L;
#pragma unroll
        for (int k = 0; k < B::R; ++k) {
            const int n0 = B::TPL * k;
            const unsigned bal = __ballot_sync(0xffffffffu, Vr[n0 + q] > thr);
            if constexpr (B::TPL == 32) {
                if (q == 0) mask[(g * L + n0) >> 5] = bal;
            } else {
                if (q == 0) reinterpret_cast<uint16_t*>(mask)[(g * L + n0) >> 4] = (uint16_t)(bal >> (t & 16));
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();
    Cx<float> v[B::R];
#pragma unroll
    for (int k = 0; k < B::R; ++k) {
        const int n = q + B::TPL * k;
        v[k] = flip(Xt[line * L + n], r + n);
    }
    big_row_forward<L>(v, Yt + line * L, tw, q, Y + g * L);
}

// a tile of column lines of one pattern: DFT, op, IDFT, in place.
// op 0: modulus projection with A (pattern b's plane at A + b * a_stride;
// vec_a: its rows 16-byte aligned); op 1: multiply by gt[f] * gt[c] (and zero
// vmax[0..nzero) for the blur pass)
template <int L, int OP, int DMODE>
__global__ void __launch_bounds__(Big<L>::NT, Big<L>::MINB) k_big_cols(Cx<float>* __restrict__ Y, const float* __restrict__ A,
                                                            uint64_t a_stride, const float* __restrict__ gtab,
                                                            const Cx<float>* __restrict__ twg,
                                                            unsigned int* __restrict__ vzero, int nzero, int vec_a) {
    constexpr int op = OP;
    using B = Big<L>;
    constexpr int CS = B::CS, AS = B::AS, LN = B::CL, NT = B::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* buf = reinterpret_cast<Cx<float>*>(smem_raw);
    Cx<float>* tw = buf + L * CS;
    float* As = reinterpret_cast<float*>(tw + B::F::TW_ENTRIES);
    float* gt = As + L * AS;
    const int t = threadIdx.x;
    int line, q;
    B::col_lane(t, line, q);
    constexpr int TILES = L / LN;
    const uint64_t b = blockIdx.x / TILES;
    const int c0 = (int)(blockIdx.x % TILES) * LN;
    Cx<float>* __restrict__ P = Y + b * (uint64_t)L * L + c0;
    stage_col_tile<L, LN, CS, AS>(buf, P, As, op == 0 ? A + b * a_stride + c0 : nullptr, L, vec_a != 0, t, NT);
    cp_async_commit();
    B::F::fill_twiddles(tw, twg, t, NT);
    if (op == 1)
        for (int i = t; i < L; i += NT) gt[i] = gtab[i];
    if (vzero && blockIdx.x == 0)
        for (int i = t; i < nzero; i += NT) vzero[i] = 0u;  // below ordered() of every float
    cp_async_wait<0>();
    __syncthreads();
    const int c = c0 + line;
    Cx<float>* col = buf + line;  // slot u of this column at col[u * CS]
    Cx<float> v[B::R], o[B::R];
#pragma unroll
    for (int k = 0; k < B::R; ++k) v[k] = col[(q + B::TPL * k) * CS];
    B::F::template natural_to_split_flat<false>(v, o, col, CS, tw, q);
#pragma unroll
    for (int i = 0; i < B::R; ++i) {
        const int f = B::pos(q, i);
        if constexpr (OP == 0)
            o[i] = data_apply(o[i], As[f * AS + line], DMODE);
        else
            o[i] = cscale(o[i], gt[f] * gt[c]);
    }
    if constexpr (!B::F::HALF) {
        // split layout in registers: the inverse runs straight from it
        B::F::template split_to_natural<true>(reinterpret_cast<Cx<float>(&)[B::F::J][B::TPL]>(o), v, col, CS, tw, q);
#pragma unroll
        for (int i = 0; i < B::R; ++i) col[(q + B::TPL * brev<B::R>(i)) * CS] = v[i];
    } else {
#pragma unroll
        for (int i = 0; i < B::R; ++i) col[B::pos(q, i) * CS] = o[i];
        __syncwarp();
#pragma unroll
        for (int k = 0; k < B::R; ++k) v[k] = col[(q + B::TPL * k) * CS];
        B::F::template natural_to_split_flat<true>(v, o, col, CS, tw, q);
#pragma unroll
        for (int i = 0; i < B::R; ++i) col[B::pos(q, i) * CS] = o[i];
    }
    __syncthreads();
    store_col_tile<L, LN, CS>(P, buf, L, t, NT);
}

enum RowsMode : int { ROWS_HIO = 0, ROWS_HIO_NEXT = 1, ROWS_HIO_MAG = 2, ROWS_BLUR = 3, ROWS_ESTIMATE = 4 };

// y = D (.) row IDFT(Y) * scale, then by mode
//   ROWS_HIO:      x <- y inside the support (and Re y >= 0 with positivity),
//                  x - beta*y elsewhere
//   ROWS_HIO_NEXT: the same, then Y <- row DFT of D (.) x (the next iteration's
//                  first pass)
//   ROWS_HIO_MAG:  the same, then Y <- row DFT of D (.) |x| (a shrinkwrap blur)
//   ROWS_BLUR:     V <- Re y; vmax[pattern] <- max(vmax, max V)
//   ROWS_ESTIMATE: x <- y inside the support, 0 elsewhere
// Y's rows arrive by asynchronous copy first, x's and the support mask's
// while the inverse transform runs.  vec_x: x rows 16-byte aligned.
template <int L, int MODE>
__global__ void __launch_bounds__(Big<L>::NT, Big<L>::MINB) k_big_rows(Cx<float>* __restrict__ Y, Cx<float>* __restrict__ x,
                                                            const uint32_t* __restrict__ mask,
                                                            float* __restrict__ vout, unsigned int* __restrict__ vmax,
                                                            const Cx<float>* __restrict__ twg, float scale, float beta,
                                                            int positivity, int vec_x) {
    constexpr int mode = MODE;
    using B = Big<L>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* Yt = reinterpret_cast<Cx<float>*>(smem_raw);
    Cx<float>* Xt = Yt + B::tile;
    Cx<float>* tw = Xt + B::tile;
    uint32_t* Mt = reinterpret_cast<uint32_t*>(tw + B::F::TW_ENTRIES);
    unsigned int* smax = Mt + B::tile / 32;
    const int t = threadIdx.x;
    int line, q;
    B::row_lane(t, line, q);
    const uint64_t g0 = (uint64_t)blockIdx.x * B::RL;
    const uint64_t b = g0 / L;
    const bool hio = mode <= ROWS_HIO_MAG;
    stage(Yt, Y + g0 * L, (uint32_t)(B::tile * 8), true, t, B::NT);
    cp_async_commit();
    if (hio) stage(Xt, x + g0 * L, (uint32_t)(B::tile * 8), vec_x, t, B::NT);
    if (hio || mode == ROWS_ESTIMATE) stage(Mt, mask + g0 * B::MW, (uint32_t)(B::tile / 8), true, t, B::NT);
    cp_async_commit();
    B::F::fill_twiddles(tw, twg, t, B::NT);
    if (t == 0) *smax = 0u;
    const uint64_t g = g0 + line;
    const int r = (int)(g % L);
    Cx<float>* yl = Yt + line * L;
    cp_async_wait<1>();  // the Y tile
    __syncthreads();
    Cx<float> v[B::R], o[B::R];
#pragma unroll
    for (int k = 0; k < B::R; ++k) v[k] = yl[q + B::TPL * k];
    B::F::template natural_to_split_flat<true>(v, o, yl, 1, tw, q);
    cp_async_wait<0>();  // x and mask tiles
    __syncthreads();
    Cx<float>* __restrict__ xr = x + g * L;
    const Cx<float>* xs = Xt + line * L;
    const uint32_t* ms = Mt + line * B::MW;
    auto inside = [&](int f) { return (ms[f >> 5] >> (f & 31)) & 1u; };
    float lmax = -INFINITY;
#pragma unroll
    for (int i = 0; i < B::R; ++i) {
        const int f = B::pos(q, i);
        const Cx<float> y = flip(cscale(o[i], scale), r + f);
        if (hio) {
            const bool keep = inside(f) && (!positivity || y.x >= 0.0f);
            const Cx<float> xn = keep ? y : merge_apply(y, xs[f], -beta, 1.0f);
            xr[f] = xn;
            // the next forward transform's input (kept in registers in the
            // split layout, else in the line's now free slots)
            const Cx<float> z =
                flip(mode == ROWS_HIO_MAG ? Cx<float>{sqrtf(fmaf(xn.x, xn.x, xn.y * xn.y)), 0.0f} : xn, r + f);
            if constexpr (!B::F::HALF)
                o[i] = z;
            else
                yl[f] = z;
        } else if (mode == ROWS_BLUR) {
            vout[g * L + f] = y.x;
            lmax = fmaxf(lmax, y.x);
        } else {
            xr[f] = inside(f) ? y : Cx<float>{0.0f, 0.0f};
        }
    }
    if (mode == ROWS_HIO_NEXT || mode == ROWS_HIO_MAG) {
        if constexpr (!B::F::HALF) {
            // split_to_natural<false> is the forward DFT of its input read as
            // a sequence indexed by the split positions: Y's row in natural order
            B::F::template split_to_natural<false>(reinterpret_cast<Cx<float>(&)[B::F::J][B::TPL]>(o), v, yl, 1, tw,
                                                   q);
            Cx<float>* __restrict__ yr = Y + g * L;
#pragma unroll
            for (int i = 0; i < B::R; ++i) yr[q + B::TPL * brev<B::R>(i)] = v[i];
        } else {
            __syncwarp();
#pragma unroll
            for (int k = 0; k < B::R; ++k) v[k] = yl[q + B::TPL * k];
            big_row_forward<L>(v, yl, tw, q, Y + g * L);
        }
    }
    if (mode == ROWS_BLUR) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
        if ((t & 31) == 0) atomicMax(smax, ordered(lmax));
        __syncthreads();
        if (t == 0) atomicMax(&vmax[b], *smax);  // all of the CTA's lines are rows of pattern b
    }
}

// The support as a bit mask over the chunk's [batch][L][L] pixels (bit k of
// word w: pixel 32 w + k); the grid-stride loops keep whole warps on one word.
// pack: mask <- (S > 0.5); unpack: S <- mask as 1 / 0; threshold: mask <-
// { v > threshold * vmax[pattern] }
__global__ void k_big_pack(const float* __restrict__ S, uint64_t s_stride, uint64_t plane, uint64_t batch,
                           uint32_t* __restrict__ mask) {
    const uint64_t total = plane * batch;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned bal = __ballot_sync(0xffffffffu, S[(i / plane) * s_stride + i % plane] > 0.5f);
        if ((threadIdx.x & 31) == 0) mask[i >> 5] = bal;
    }
}

__global__ void k_big_unpack(const uint32_t* __restrict__ mask, float* __restrict__ S, uint64_t s_stride,
                             uint64_t plane, uint64_t batch) {
    const uint64_t total = plane * batch;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x)
        S[(i / plane) * s_stride + i % plane] = ((mask[i >> 5] >> (i & 31)) & 1u) ? 1.0f : 0.0f;
}

__global__ void k_big_threshold(const float* __restrict__ v, const unsigned int* __restrict__ vmax,
                                uint32_t* __restrict__ mask, uint64_t plane, uint64_t batch, float threshold) {
    const uint64_t total = plane * batch;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned bal = __ballot_sync(0xffffffffu, v[i] > threshold * unordered(vmax[i / plane]));
        if ((threadIdx.x & 31) == 0) mask[i >> 5] = bal;
    }
}

template <int L>
cudaError_t big_set_smem() {
    using B = Big<L>;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_big_rows_fwd<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)B::row_smem())) != cudaSuccess)
        return e;
    for (auto k : {k_big_rows<L, ROWS_HIO>, k_big_rows<L, ROWS_HIO_NEXT>, k_big_rows<L, ROWS_HIO_MAG>,
                   k_big_rows<L, ROWS_BLUR>, k_big_rows<L, ROWS_ESTIMATE>})
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B::row_smem())) !=
            cudaSuccess)
            return e;
    if ((e = cudaFuncSetAttribute(k_big_cols<L, 0, DATA_SKIP_ZERO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)B::col_smem())) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_big_cols<L, 0, DATA_ALWAYS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)B::col_smem())) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_big_cols<L, 1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B::col_smem());
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// all iterations of one chunk of `nb` patterns: per iteration one column
// pass and one row pass (the row pass ends with the next iteration's forward
// row transform); a shrinkwrap update adds a blur column pass, a blur row
// pass and a forward row pass that also writes the new support mask
template <int L>
cudaError_t big_chunk(const HioArgs& a, uint64_t b0, uint64_t nb, const Cx<float>* tw, Cx<float>* Y, float* V,
                      unsigned int* vmax, uint32_t* mask, cudaStream_t st) {
    using B = Big<L>;
    constexpr int NT = B::NT;
    const uint64_t plane = (uint64_t)L * L;
    Cx<float>* x = (Cx<float>*)a.x + b0 * plane;
    const float* A = (const float*)a.A + b0 * a.a_stride;
    float* S = (float*)a.S + b0 * a.s_stride;
    const int vx = aligned16(a.x), va = aligned16(a.A) && a.a_stride % 4 == 0;
    const unsigned row_ctas = (unsigned)(nb * L / B::RL);
    const unsigned col_ctas = (unsigned)(nb * (L / B::CL));
    const unsigned ew = ew_grid(nb * plane, 256);
    const size_t rs = B::row_smem(), cs = B::col_smem();
    const float scale = 1.0f / (float)plane, beta = (float)a.beta, thr = (float)a.threshold;
    const bool est = a.estimate != nullptr;
    auto cols = [&](int op, const float* gtab, unsigned int* vz) {
        if (op == 1)
            k_big_cols<L, 1, 0><<<col_ctas, NT, cs, st>>>(Y, A, a.a_stride, gtab, tw, vz, (int)nb, va);
        else if (a.data_mode == DATA_ALWAYS)
            k_big_cols<L, 0, DATA_ALWAYS><<<col_ctas, NT, cs, st>>>(Y, A, a.a_stride, gtab, tw, vz, (int)nb, va);
        else
            k_big_cols<L, 0, DATA_SKIP_ZERO><<<col_ctas, NT, cs, st>>>(Y, A, a.a_stride, gtab, tw, vz, (int)nb, va);
    };
    auto rows = [&](Cx<float>* dst, int mode, int pos, int vdst) {
        switch (mode) {
            case ROWS_HIO:
                k_big_rows<L, ROWS_HIO><<<row_ctas, NT, rs, st>>>(Y, dst, mask, V, vmax, tw, scale, beta, pos, vdst);
                break;
            case ROWS_HIO_NEXT:
                k_big_rows<L, ROWS_HIO_NEXT>
                    <<<row_ctas, NT, rs, st>>>(Y, dst, mask, V, vmax, tw, scale, beta, pos, vdst);
                break;
            case ROWS_HIO_MAG:
                k_big_rows<L, ROWS_HIO_MAG>
                    <<<row_ctas, NT, rs, st>>>(Y, dst, mask, V, vmax, tw, scale, beta, pos, vdst);
                break;
            case ROWS_BLUR:
                k_big_rows<L, ROWS_BLUR><<<row_ctas, NT, rs, st>>>(Y, dst, mask, V, vmax, tw, scale, beta, pos, vdst);
                break;
            default:
                k_big_rows<L, ROWS_ESTIMATE>
                    <<<row_ctas, NT, rs, st>>>(Y, dst, mask, V, vmax, tw, scale, beta, pos, vdst);
                break;
        }
    };
    k_big_pack<<<ew, 256, 0, st>>>(S, a.s_stride, plane, nb, mask);
    k_big_rows_fwd<L><<<row_ctas, NT, rs, st>>>(x, Y, tw, nullptr, nullptr, mask, thr, vx);
    uint64_t launches = 2;
    int update = 0;
    for (int it = 0; it < a.iters; ++it) {
        const bool last = (it + 1 == a.iters);
        const bool sw = a.sw_every > 0 && a.blur && (it + 1) % a.sw_every == 0;
        cols(0, nullptr, nullptr);
        if (!sw) {
            rows(x, (last && !est) ? ROWS_HIO : ROWS_HIO_NEXT, a.positivity, vx);
            launches += 2;
            continue;
        }
        rows(x, ROWS_HIO_MAG, a.positivity, vx);
        cols(1, (const float*)a.blur + (size_t)update * L, vmax);
        rows(x, ROWS_BLUR, 0, vx);
        launches += 4;
        ++update;
        if (last && !est)
            k_big_threshold<<<ew, 256, 0, st>>>(V, vmax, mask, plane, nb, thr);
        else
            k_big_rows_fwd<L><<<row_ctas, NT, rs, st>>>(x, Y, tw, V, vmax, mask, thr, vx);
        ++launches;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (est) {
        // S (.) P_M(x): Y holds the forward row transform of the final x
        cols(0, nullptr, nullptr);
        rows((Cx<float>*)a.estimate + b0 * plane, ROWS_ESTIMATE, 0, 0);
        launches += 2;
    }
    k_big_unpack<<<ew, 256, 0, st>>>(mask, S, a.s_stride, plane, nb);
    count_launches(launches + 1);
    return cudaGetLastError();
}

template <int L>
cudaError_t big_hio(const HioArgs& a, const void* tw, void* Y, void* V, unsigned int* vmax, uint32_t* mask,
                    uint64_t chunk, cudaStream_t st) {
    cudaError_t e = big_set_smem<L>();
    if (e != cudaSuccess) return e;
    for (uint64_t b0 = 0; b0 < a.batch; b0 += chunk) {
        const uint64_t nb = (a.batch - b0 < chunk) ? a.batch - b0 : chunk;
        if ((e = big_chunk<L>(a, b0, nb, (const Cx<float>*)tw, (Cx<float>*)Y, (float*)V, vmax, mask, st)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

}  // namespace

bool hio_large_supported(bool dbl, uint64_t M, uint64_t N) { return !dbl && M == N && (M == 256 || M == 512); }

cudaError_t launch_hio_large(const HioArgs& a, const void* tw, void* Y, void* V, unsigned int* vmax, uint32_t* mask,
                             uint64_t chunk, cudaStream_t st) {
    if (!hio_large_supported(false, a.M, a.N) || chunk == 0) return cudaErrorInvalidValue;
    if (a.batch == 0 || (a.iters <= 0 && !a.estimate)) return cudaSuccess;
    switch (a.M) {
        case 256: return big_hio<256>(a, tw, Y, V, vmax, mask, chunk, st);
        case 512: return big_hio<512>(a, tw, Y, V, vmax, mask, chunk, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cpra_b200
