// Difference-map iterations (the reference's 12-call iteration,
// src/CPRA_MKL.cpp:94-110) for 256 x 256 and 512 x 512 float planes, whose
// plane is too large for one CTA, as line passes over the batch:
//   first   per row: carousel mix and t1 = t2 = x when the launch starts an
//           angle, t2' = a2*x + b2*S(t2), then the forward row DFTs of
//           D (.) t1 and D (.) t2' into Y = [batch][2][L][L]     k_dml_first
//   columns per column of both planes: forward column DFT, DataConstraint(A),
//           inverse column DFT                                   k_dml_cols
//   rows    per row: inverse row DFTs (times D/(MN)) give P_M(t1), P_M(t2');
//           t1 <- S(a1*x + b1*P_M(t1)), t2 <- P_M(t2'),
//           x <- a4*t2 + b4*(a3*t1 + b3*x); then, unless it is the launch's
//           last iteration, the next iteration's forward row DFTs of t1 and
//           t2' = a2*x + b2*S(t2)                                k_dml_rows
// so an iteration is one column pass and one row pass, and t1, t2 are written
// only by the last one.  D = (-1)^(row + col) folds the fftshifts; the two
// around DataConstraint cancel (it commutes with the sign pattern).
//
// Every 1D transform is LineFFT::natural_to_split_flat with the per-operator
// axis passes' split (line_pass.cuh LineGeom: 16 threads per line at 256, 32
// at 512), fed in natural order,
// and the element-wise steps are ops_ew.cuh's, so a launch writes the same
// bits as the 12 per-operator calls per iteration.  SpaceConstraint is the
// threshold form (MKL_Impl.inl:70-84) through a bit mask of the support.
#include "cpra_internal.h"
#include "line_pass.cuh"
#include "ops_ew.cuh"

namespace cpra_b200 {
namespace {

template <int L>
struct DmLP : LineGeom<L> {
    using G = LineGeom<L>;
    using F = typename G::F;
    static constexpr int TPL = G::TPL, R = G::R, NT = G::THREADS;
    static constexpr int RL = G::ROW_LINES, CL = G::COL_LINES, CS = G::CS, AS = G::AS;
    static constexpr int MW = L / 32;  // mask words per row
    static constexpr size_t tile = G::row_tile;
    // rows: Y tile (Y1's rows, then each line's Y2 row), x tile, twiddles, mask tile
    static constexpr size_t row_smem() { return sizeof(Cx<float>) * (2 * tile + F::TW_ENTRIES) + tile / 8; }
    static constexpr size_t col_smem() {
        return sizeof(Cx<float>) * ((size_t)L * CS + F::TW_ENTRIES) + sizeof(float) * (size_t)L * AS;
    }
};

struct DmlDev {
    Cx<float>* x;
    Cx<float>* t1;
    Cx<float>* t2;
    const Cx<float>* xprev;
    const Cx<float>* xnext;
    int mix, init_from_x;
    const float* A;
    uint64_t a_stride;
    const uint32_t* mask;  // support bits (set = kept), one plane per pattern or one shared
    uint64_t mask_stride;  // words between patterns' planes (0: shared)
    Cx<float>* Y;          // [batch][2][L][L]
    const Cx<float>* tw;
    float scale, a1, b1, a2, b2, a3, b3, a4, b4;
    int data_mode, vec_x, vec_a;
};

__device__ __forceinline__ Cx<float> keep_re(Cx<float> z, uint32_t bit) { return {bit ? z.x : 0.0f, 0.0f}; }

// support mask <- !(S <= 0.9f) (SpaceConstraint keeps the real part there)
__global__ void k_dml_pack(const float* __restrict__ S, uint64_t s_stride, uint64_t plane, uint64_t planes,
                           uint32_t* __restrict__ mask) {
    const uint64_t total = plane * planes;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned bal = __ballot_sync(0xffffffffu, !space_zero(S[(i / plane) * s_stride + i % plane]));
        if ((threadIdx.x & 31) == 0) mask[i >> 5] = bal;
    }
}

template <int L>
__global__ void __launch_bounds__(DmLP<L>::NT, 3) k_dml_first(const DmlDev p) {
    using B = DmLP<L>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* scratch = reinterpret_cast<Cx<float>*>(smem_raw);
    Cx<float>* tw = scratch + B::tile;
    const int t = threadIdx.x;
    int line, q;
    B::row_lane(t, line, q);
    B::F::fill_twiddles(tw, p.tw, t, B::NT);
    const uint64_t g = (uint64_t)blockIdx.x * B::RL + line, b = g / L;
    const int r = (int)(g % L);
    // distinct buffers (x is the angle's own plane, its neighbours' are
    // others), so the loads of later elements need not wait for x's stores
    Cx<float>* __restrict__ X = p.x + g * L;
    const Cx<float>* __restrict__ T1 = p.t1 + g * L;
    const Cx<float>* __restrict__ T2 = p.t2 + g * L;
    const Cx<float>* __restrict__ XP = p.xprev ? p.xprev + g * L : nullptr;
    const Cx<float>* __restrict__ XN = p.xnext ? p.xnext + g * L : nullptr;
    const uint32_t* __restrict__ mr = p.mask + b * p.mask_stride + (uint64_t)r * B::MW;
    __syncthreads();  // twiddle table
#pragma unroll 1
    for (int pl = 0; pl < 2; ++pl) {
        Cx<float> v[B::R], o[B::R];
#pragma unroll
        for (int k = 0; k < B::R; ++k) {
            const int n = q + B::TPL * k;
            Cx<float> xv = X[n];
            Cx<float> z;
            if (pl == 0) {
                if (p.init_from_x) {
                    // the angle's start: carousel mix of x (src/CPRA_MKL.cpp:64-76), then t1 = x
                    if (p.mix == MIX_FIRST) {
                        xv = merge_apply(XN[n], xv, 0.5f, 0.5f);
                    } else if (p.mix == MIX_LAST) {
                        xv = merge_apply(XP[n], xv, 0.5f, 0.5f);
                    } else if (p.mix == MIX_MIDDLE) {
                        xv = merge_apply(XP[n], xv, 0.5f, 0.0f);
                        xv = merge_apply(XN[n], xv, 0.5f, 1.0f);
                    }
                    if (p.mix != MIX_NONE) X[n] = xv;
                    z = xv;
                } else {
                    z = T1[n];
                }
            } else {
                const uint32_t bit = (mr[n >> 5] >> (n & 31)) & 1u;
                z = merge_apply(xv, keep_re(p.init_from_x ? xv : T2[n], bit), p.a2, p.b2);
            }
            v[k] = flip(z, r + n);
        }
        B::F::template natural_to_split_flat<false>(v, o, scratch + line * L, 1, tw, q);
        Cx<float>* __restrict__ yr = p.Y + ((2 * b + pl) * (uint64_t)L + r) * L;
#pragma unroll
        for (int i = 0; i < B::R; ++i) yr[B::pos(q, i)] = o[i];
    }
}

// a tile of column lines of one plane (2 per pattern): forward column DFT,
// DataConstraint with the pattern's A (mode DMODE), inverse column DFT, in place
template <int L, int DMODE>
__global__ void __launch_bounds__(DmLP<L>::NT, 3) k_dml_cols(const DmlDev p) {
    using B = DmLP<L>;
    constexpr int CS = B::CS, AS = B::AS, LN = B::CL, NT = B::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* buf = reinterpret_cast<Cx<float>*>(smem_raw);
    Cx<float>* tw = buf + L * CS;
    float* As = reinterpret_cast<float*>(tw + B::F::TW_ENTRIES);
    const int t = threadIdx.x;
    int line, q;
    B::col_lane(t, line, q);
    constexpr int TILES = L / LN;
    const uint64_t pl = blockIdx.x / TILES, b = pl / 2;
    const int c0 = (int)(blockIdx.x % TILES) * LN;
    Cx<float>* __restrict__ P = p.Y + pl * (uint64_t)L * L + c0;
    stage_col_tile<L, LN, CS, AS>(buf, P, As, p.A + b * p.a_stride + c0, L, p.vec_a != 0, t, NT);
    cp_async_commit();
    B::F::fill_twiddles(tw, p.tw, t, NT);
    cp_async_wait<0>();
    __syncthreads();
    Cx<float>* col = buf + line;  // slot u of this column at col[u * CS]
    Cx<float> v[B::R], o[B::R];
#pragma unroll
    for (int k = 0; k < B::R; ++k) v[k] = col[(q + B::TPL * k) * CS];
    B::F::template natural_to_split_flat<false>(v, o, col, CS, tw, q);
#pragma unroll
    for (int i = 0; i < B::R; ++i) {
        const int f = B::pos(q, i);
        col[f * CS] = data_apply(o[i], As[f * AS + line], DMODE);
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < B::R; ++k) v[k] = col[(q + B::TPL * k) * CS];
    B::F::template natural_to_split_flat<true>(v, o, col, CS, tw, q);
#pragma unroll
    for (int i = 0; i < B::R; ++i) col[B::pos(q, i) * CS] = o[i];
    __syncthreads();
    store_col_tile<L, LN, CS>(P, buf, L, t, NT);
}

// the rest of an iteration and, unless `last`, the next one's forward rows.
// t1's half (inverse, update, next forward into Y1) completes first; then each
// line's threads copy that line's row of Y2 into the slots it has freed, so a
// CTA stages two tiles (Y, x), not three.
template <int L>
__global__ void __launch_bounds__(DmLP<L>::NT, 3) k_dml_rows(const DmlDev p, int last) {
    using B = DmLP<L>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* Yt = reinterpret_cast<Cx<float>*>(smem_raw);
    Cx<float>* Xt = Yt + B::tile;
    Cx<float>* tw = Xt + B::tile;
    uint32_t* Mt = reinterpret_cast<uint32_t*>(tw + B::F::TW_ENTRIES);
    const int t = threadIdx.x;
    int line, q;
    B::row_lane(t, line, q);
    const uint64_t g0 = (uint64_t)blockIdx.x * B::RL, b = g0 / L;
    const int r0 = (int)(g0 % L);
    Cx<float>* Y1 = p.Y + (2 * b * (uint64_t)L + r0) * L;
    Cx<float>* Y2 = Y1 + (uint64_t)L * L;
    stage(Yt, Y1, (uint32_t)(B::tile * 8), true, t, B::NT);
    cp_async_commit();
    stage(Xt, p.x + g0 * L, (uint32_t)(B::tile * 8), p.vec_x, t, B::NT);
    stage(Mt, p.mask + b * p.mask_stride + (uint64_t)r0 * B::MW, (uint32_t)(B::tile / 8), true, t, B::NT);
    cp_async_commit();
    B::F::fill_twiddles(tw, p.tw, t, B::NT);
    const int r = r0 + line;
    const uint64_t row = g0 + line;
    Cx<float>* yl = Yt + line * L;
    Cx<float>* xs = Xt + line * L;
    const uint32_t* ms = Mt + line * B::MW;
    auto bit = [&](int f) { return (ms[f >> 5] >> (f & 31)) & 1u; };
    Cx<float> v[B::R], o[B::R];
    // the line's natural-order slots (D-flipped) through the forward row
    // transform into the global row yg
    auto forward_row = [&](Cx<float>* __restrict__ yg) {
#pragma unroll
        for (int k = 0; k < B::R; ++k) v[k] = flip(yl[q + B::TPL * k], r + q + B::TPL * k);
        B::F::template natural_to_split_flat<false>(v, o, yl, 1, tw, q);
#pragma unroll
        for (int i = 0; i < B::R; ++i) yg[B::pos(q, i)] = o[i];
    };

    // t1 <- S(a1*x + b1*P_M(t1)); x1 = a3*t1 + b3*x (kept in the x tile)
    cp_async_wait<1>();
    __syncthreads();
#pragma unroll
    for (int k = 0; k < B::R; ++k) v[k] = yl[q + B::TPL * k];
    B::F::template natural_to_split_flat<true>(v, o, yl, 1, tw, q);
    cp_async_wait<0>();
    __syncthreads();
#pragma unroll
    for (int i = 0; i < B::R; ++i) {
        const int f = B::pos(q, i);
        const Cx<float> pm = flip(cscale(o[i], p.scale), r + f);
        const Cx<float> xv = xs[f];
        const Cx<float> t1n = keep_re(merge_apply(xv, pm, p.a1, p.b1), bit(f));
        xs[f] = merge_apply(t1n, xv, p.a3, p.b3);
        yl[f] = t1n;
        if (last) p.t1[row * L + f] = t1n;
    }
    __syncwarp();
    if (!last) forward_row(Y1 + (uint64_t)line * L);
    // the line's row of Y2 into its slots (this line's threads only)
    stage(yl, Y2 + (uint64_t)line * L, (uint32_t)(L * 8), true, q, B::TPL);
    cp_async_commit();
    cp_async_wait<0>();
    __syncwarp();
    // t2 <- P_M(t2'); x <- a4*t2 + b4*x1; the next t2' = a2*x + b2*S(t2)
#pragma unroll
    for (int k = 0; k < B::R; ++k) v[k] = yl[q + B::TPL * k];
    B::F::template natural_to_split_flat<true>(v, o, yl, 1, tw, q);
#pragma unroll
    for (int i = 0; i < B::R; ++i) {
        const int f = B::pos(q, i);
        const Cx<float> t2n = flip(cscale(o[i], p.scale), r + f);
        const Cx<float> xn = merge_apply(t2n, xs[f], p.a4, p.b4);
        p.x[row * L + f] = xn;
        if (last)
            p.t2[row * L + f] = t2n;
        else
            yl[f] = merge_apply(xn, keep_re(t2n, bit(f)), p.a2, p.b2);
    }
    if (last) return;
    __syncwarp();
    forward_row(Y2 + (uint64_t)line * L);
}

template <int L>
cudaError_t dml_launch(const DmArgs& a, const void* tw, void* Y, uint32_t* mask, cudaStream_t st) {
    using B = DmLP<L>;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_dml_first<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)B::row_smem())) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_dml_rows<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)B::row_smem())) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_dml_cols<L, DATA_SKIP_ZERO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)B::col_smem())) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_dml_cols<L, DATA_ALWAYS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)B::col_smem())) != cudaSuccess)
        return e;
    const uint64_t plane = (uint64_t)L * L;
    DmlDev d;
    d.x = (Cx<float>*)a.x;
    d.t1 = (Cx<float>*)a.t1;
    d.t2 = (Cx<float>*)a.t2;
    d.xprev = (const Cx<float>*)a.xprev;
    d.xnext = (const Cx<float>*)a.xnext;
    d.mix = a.mix;
    d.init_from_x = a.init_from_x;
    d.A = (const float*)a.A;
    d.a_stride = a.a_stride;
    d.mask = mask;
    d.mask_stride = a.s_stride ? plane / 32 : 0;
    d.Y = (Cx<float>*)Y;
    d.tw = (const Cx<float>*)tw;
    d.scale = 1.0f / (float)plane;  // DFTI_BACKWARD_SCALE (include/MKL_Impl.hpp:40)
    d.a1 = (float)a.c.a1;
    d.b1 = (float)a.c.b1;
    d.a2 = (float)a.c.a2;
    d.b2 = (float)a.c.b2;
    d.a3 = (float)a.c.a3;
    d.b3 = (float)a.c.b3;
    d.a4 = (float)a.c.a4;
    d.b4 = (float)a.c.b4;
    d.data_mode = a.data_mode;
    d.vec_x = (reinterpret_cast<uintptr_t>(a.x) & 15u) == 0;
    d.vec_a = (reinterpret_cast<uintptr_t>(a.A) & 15u) == 0 && a.a_stride % 4 == 0;
    const uint64_t planes = a.s_stride ? a.batch : 1;
    k_dml_pack<<<ew_grid(planes * plane, 256), 256, 0, st>>>((const float*)a.S, a.s_stride, plane, planes, mask);
    const unsigned row_ctas = (unsigned)(a.batch * L / B::RL);
    const unsigned col_ctas = (unsigned)(2 * a.batch * (L / B::CL));
    k_dml_first<L><<<row_ctas, B::NT, B::row_smem(), st>>>(d);
    for (int it = 0; it < a.iters; ++it) {
        if (a.data_mode == DATA_ALWAYS)
            k_dml_cols<L, DATA_ALWAYS><<<col_ctas, B::NT, B::col_smem(), st>>>(d);
        else
            k_dml_cols<L, DATA_SKIP_ZERO><<<col_ctas, B::NT, B::col_smem(), st>>>(d);
        k_dml_rows<L><<<row_ctas, B::NT, B::row_smem(), st>>>(d, it + 1 == a.iters ? 1 : 0);
    }
    count_launches(2 + 2 * (uint64_t)a.iters);
    return cudaGetLastError();
}

}  // namespace

namespace {
template <int L>
int dml_occupancy() {
    using B = DmLP<L>;
    if (cudaFuncSetAttribute(k_dml_rows<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B::row_smem()) !=
        cudaSuccess)
        return 1;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_dml_rows<L>, B::NT, B::row_smem()) != cudaSuccess || n < 1)
        return 1;
    return n;
}
}  // namespace

int dm_large_ctas_per_sm(uint64_t M) { return M == 256 ? dml_occupancy<256>() : M == 512 ? dml_occupancy<512>() : 1; }

uint64_t dm_large_row_ctas(uint64_t M, uint64_t batch) {
    return M == 256 ? batch * 256 / DmLP<256>::RL : M == 512 ? batch * 512 / DmLP<512>::RL : batch;
}

bool dm_large_supported(bool dbl, uint64_t M, uint64_t N, int space_mode) {
    return !dbl && M == N && (M == 256 || M == 512) && space_mode == SPACE_THRESHOLD;
}

uint64_t dm_large_scratch_bytes(uint64_t M, uint64_t N, uint64_t batch, uint64_t s_stride) {
    const uint64_t plane = M * N;
    return 2 * batch * plane * 8 + (s_stride ? batch : 1) * plane / 8;
}

cudaError_t launch_dm_large(const DmArgs& a, const void* tw, void* scratch, cudaStream_t st) {
    if (!dm_large_supported(false, a.M, a.N, a.space_mode)) return cudaErrorInvalidValue;
    if (a.batch == 0 || a.iters <= 0) return cudaSuccess;
    if (a.s_stride != 0 && a.s_stride != a.M * a.N) return cudaErrorInvalidValue;
    char* w = static_cast<char*>(scratch);
    uint32_t* mask = reinterpret_cast<uint32_t*>(w + 2 * a.batch * a.M * a.N * 8);
    switch (a.M) {
        case 256: return dml_launch<256>(a, tw, w, mask, st);
        case 512: return dml_launch<512>(a, tw, w, mask, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cpra_b200
