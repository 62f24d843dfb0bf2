// Fused difference-map iterations: the reference's 12-call iteration
// (src/CPRA_MKL.cpp:94-110)
//   t1 <- Forward2D; DataConstraint(A); Backward2D; t1 <- a1*x + b1*t1; SpaceConstraint(S)
//   t2 <- SpaceConstraint(S); t2 <- a2*x + b2*t2; Forward2D; DataConstraint(A); Backward2D
//   x  <- a3*t1 + b3*x;  x <- a4*t2 + b4*x
// as one kernel with one CTA per pattern.  The pattern's plane stays in shared
// memory for all four transforms; t1 (real after SpaceConstraint) stays in
// shared memory across iterations; x, t2, A and S are read from global memory
// (L2) where each step needs them.  The fftshifts cancel in pairs around the
// modulus step (DataConstraint commutes with the (-1)^(i+j) sign pattern), so
// only the sign flips on the input of each forward and the output of each
// inverse transform remain.
//
// The arithmetic is the per-operator kernels' arithmetic step for step
// (Plane<> passes, ops_ew.cuh operators), so one launch with `iters`
// iterations writes the same bits as 12*iters per-operator calls.
#include "cpra_internal.h"
#include "fft2d_cta.cuh"
#include "ops_ew.cuh"

namespace cpra_b200 {

namespace {

struct DmDev {
    Cx<float>* x;
    Cx<float>* t1;
    Cx<float>* t2;
    const float* A;
    uint64_t a_stride;
    const float* S;
    uint64_t s_stride;
    const Cx<float>* tw;
    float scale;
    float a1, b1, a2, b2, a3, b3, a4, b4;
    int iters, space_mode, data_mode;
};

// Shared memory of one CTA: the plane buffer, t1's real part (row pitch L + 4
// so that the 4-byte accesses of a warp's 8 rows fall on distinct banks), the
// twiddle table, and the support as a bit mask (SpaceConstraint's threshold
// test, evaluated once per launch: bit set where the value is kept).
template <int L>
struct DmPlan {
    using P = Plane<float, L>;
    static constexpr int T1S = L + 4;
    static constexpr int MASK_WORDS = L * L / 32;
    static constexpr size_t t1_bytes() { return sizeof(float) * (size_t)L * T1S; }
    static constexpr size_t smem_bytes() {
        return P::buf_bytes() + t1_bytes() + P::tw_bytes() + sizeof(uint32_t) * MASK_WORDS;
    }
};

__device__ __forceinline__ bool mask_keep(const uint32_t* mask, int idx) { return (mask[idx >> 5] >> (idx & 31)) & 1u; }

// column forward transform, modulus projection, column inverse transform
template <int L>
__device__ __forceinline__ void modulus_columns(Cx<float>* buf, const Cx<float>* tw, const float* __restrict__ A,
                                                int c, int q, int data_mode) {
    using P = Plane<float, L>;
    Cx<float> o[P::J][P::TPL];
    P::template col_from_buf<false>(o, buf, tw, c, q);
#pragma unroll
    for (int j = 0; j < P::J; ++j)
#pragma unroll
        for (int s = 0; s < P::TPL; ++s) {
            const int f = P::split_pos(q, j, s);
            o[j][s] = data_apply(o[j][s], A[f * L + c], data_mode);
        }
    P::template col_to_buf<true>(o, buf, tw, c, q);
}

template <int L>
__global__ void __launch_bounds__(4 * L, 1) k_dm(const DmDev p) {
    using P = Plane<float, L>;
    using D = DmPlan<L>;
    constexpr int T1S = D::T1S;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<float>* buf = reinterpret_cast<Cx<float>*>(smem_raw);
    float* t1r = reinterpret_cast<float*>(smem_raw + P::buf_bytes());
    Cx<float>* tw = reinterpret_cast<Cx<float>*>(smem_raw + P::buf_bytes() + D::t1_bytes());
    uint32_t* mask = reinterpret_cast<uint32_t*>(smem_raw + P::buf_bytes() + D::t1_bytes() + P::tw_bytes());
    const int t = threadIdx.x, line = t >> 2, q = t & 3;
    P::F::fill_twiddles(tw, p.tw, t, P::NT);
    const size_t base = (size_t)blockIdx.x * L * L;
    Cx<float>* __restrict__ X = p.x + base;
    Cx<float>* __restrict__ T1 = p.t1 + base;
    Cx<float>* __restrict__ T2 = p.t2 + base;
    const float* __restrict__ A = p.A + blockIdx.x * p.a_stride;
    const float* __restrict__ S = p.S + blockIdx.x * p.s_stride;
    const bool use_mask = (p.space_mode == SPACE_THRESHOLD);
    if (use_mask) {
        for (int i = t; i < L * L; i += P::NT) {
            const unsigned keep = __ballot_sync(0xffffffffu, !space_zero(S[i]));
            if ((i & 31) == 0) mask[i >> 5] = keep;
        }
    }
    // SpaceConstraint of element idx, from the mask or the support plane
    auto space = [&](Cx<float> z, int idx) -> Cx<float> {
        if (use_mask) return {mask_keep(mask, idx) ? z.x : 0.0f, 0.0f};
        return space_apply(z, S[idx], p.space_mode);
    };
    __syncthreads();

    for (int it = 0; it < p.iters; ++it) {
        const bool last = (it == p.iters - 1);
        // ---- t1 <- S( a1*x + b1*Backward2D(DataConstraint(Forward2D(t1))) )
        {
            Cx<float> v[P::R];
#pragma unroll
            for (int k = 0; k < P::R; ++k) {
                const int n = q + P::TPL * k;
                const int idx = line * L + n;
                const Cx<float> z = (it == 0) ? T1[idx] : Cx<float>{t1r[line * T1S + n], 0.0f};
                v[k] = csign(z, line + n);
            }
            P::template rows_to_buf<false>(v, buf, tw, line, q);
        }
        __syncthreads();
        modulus_columns<L>(buf, tw, A, line, q, p.data_mode);
        __syncthreads();
        {
            Cx<float> o[P::J][P::TPL];
            P::template row_from_buf<true>(o, buf, tw, line, q);
#pragma unroll
            for (int j = 0; j < P::J; ++j)
#pragma unroll
                for (int s = 0; s < P::TPL; ++s) {
                    const int f = P::split_pos(q, j, s);
                    const int idx = line * L + f;
                    const Cx<float> val = csign(cscale(o[j][s], p.scale), line + f);
                    Cx<float> m = merge_apply(X[idx], val, p.a1, p.b1);
                    m = space(m, idx);
                    t1r[line * T1S + f] = m.x;
                    if (last) T1[idx] = m;
                }
        }
        __syncthreads();
        // ---- t2 <- Backward2D(DataConstraint(Forward2D( a2*x + b2*S(t2) )))
        {
            Cx<float> v[P::R];
#pragma unroll
            for (int k = 0; k < P::R; ++k) {
                const int n = q + P::TPL * k;
                const int idx = line * L + n;
                Cx<float> z = space(T2[idx], idx);
                z = merge_apply(X[idx], z, p.a2, p.b2);
                v[k] = csign(z, line + n);
            }
            P::template rows_to_buf<false>(v, buf, tw, line, q);
        }
        __syncthreads();
        modulus_columns<L>(buf, tw, A, line, q, p.data_mode);
        __syncthreads();
        {
            Cx<float> o[P::J][P::TPL];
            P::template row_from_buf<true>(o, buf, tw, line, q);
#pragma unroll
            for (int j = 0; j < P::J; ++j)
#pragma unroll
                for (int s = 0; s < P::TPL; ++s) {
                    const int f = P::split_pos(q, j, s);
                    const int idx = line * L + f;
                    const Cx<float> t2n = csign(cscale(o[j][s], p.scale), line + f);
                    T2[idx] = t2n;
                    const Cx<float> x1 = merge_apply(Cx<float>{t1r[line * T1S + f], 0.0f}, X[idx], p.a3, p.b3);
                    X[idx] = merge_apply(t2n, x1, p.a4, p.b4);
                }
        }
        __syncthreads();
    }
}

template <int L>
cudaError_t dm_launch(const DmArgs& a, const void* tw, cudaStream_t st) {
    DmDev d;
    d.x = (Cx<float>*)a.x;
    d.t1 = (Cx<float>*)a.t1;
    d.t2 = (Cx<float>*)a.t2;
    d.A = (const float*)a.A;
    d.a_stride = a.a_stride;
    d.S = (const float*)a.S;
    d.s_stride = a.s_stride;
    d.tw = (const Cx<float>*)tw;
    d.scale = 1.0f / (float)(a.M * a.N);
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
    cudaError_t e = cudaFuncSetAttribute(k_dm<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_dm<L><<<(unsigned)a.batch, 4 * L, smem, st>>>(d);
    count_launches();
    return cudaGetLastError();
}

}  // namespace

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
