// Element-wise operators of the CpraImpl<T> interface and the reductions and
// interpolations around them.  All are grid-stride kernels sized to whole
// waves over the SMs.  Constraint planes are broadcast over the batch the way
// the reference indexes them, element i using plane element i % (num/batch)
// (include/detail/MKL_Impl.inl:83,98,121): each thread keeps one plane value
// in a register and applies it to every repetition, so a plane is read once.
#include "cpra_internal.h"
#include "angle_table.cuh"
#include "ops_ew.cuh"

#include <cmath>

namespace cpra_b200 {

namespace {

constexpr int EW_THREADS = 256;

__device__ __forceinline__ uint64_t gtid() { return blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

// Broadcast kernels: blockIdx.x walks the plane, blockIdx.y a chunk of
// `reps_per_y` repetitions (element i = r * plane + j), so that the grid covers
// the whole batch while each thread keeps its plane value in a register.
template <typename T>
__global__ void k_space(Cx<T>* __restrict__ x, const T* __restrict__ s, uint64_t num, uint64_t plane,
                        uint64_t reps_per_y, int mode) {
    const uint64_t r0 = blockIdx.y * reps_per_y;
    for (uint64_t j = gtid(); j < plane; j += gstride()) {
        const T sv = s[j];
        for (uint64_t r = r0, i = r0 * plane + j; r < r0 + reps_per_y && i < num; ++r, i += plane)
            x[i] = space_apply(x[i], sv, mode);
    }
}

template <typename T>
__global__ void k_data_real(Cx<T>* __restrict__ x, const T* __restrict__ a, uint64_t num, uint64_t plane,
                            uint64_t reps_per_y, int mode) {
    const uint64_t r0 = blockIdx.y * reps_per_y;
    for (uint64_t j = gtid(); j < plane; j += gstride()) {
        const T av = a[j];
        for (uint64_t r = r0, i = r0 * plane + j; r < r0 + reps_per_y && i < num; ++r, i += plane)
            x[i] = data_apply(x[i], av, mode);
    }
}

template <typename T>
__global__ void k_data_complex(Cx<T>* __restrict__ x, const Cx<T>* __restrict__ c, uint64_t num, uint64_t plane,
                               uint64_t reps_per_y) {
    const uint64_t r0 = blockIdx.y * reps_per_y;
    for (uint64_t j = gtid(); j < plane; j += gstride()) {
        const Cx<T> cv = c[j];
        for (uint64_t r = r0, i = r0 * plane + j; r < r0 + reps_per_y && i < num; ++r, i += plane)
            x[i] = data_apply_complex(x[i], cv);
    }
}

// grid of a broadcast kernel: x covers the plane (capped at a wave of CTAs),
// y splits the repetitions so that the whole grid is about 8 CTAs per SM
struct BroadcastGrid {
    dim3 grid;
    uint64_t reps_per_y;
};
BroadcastGrid broadcast_grid(uint64_t num, uint64_t plane) {
    const uint64_t reps = (num + plane - 1) / plane;
    const uint64_t target = (uint64_t)sm_count() * 8;
    const uint64_t gx = ew_grid(plane, EW_THREADS);
    uint64_t gy = target / gx;
    if (gy < 1) gy = 1;
    if (gy > reps) gy = reps;
    if (gy > 65535) gy = 65535;
    const uint64_t per = (reps + gy - 1) / gy;
    gy = (reps + per - 1) / per;
    return {dim3((unsigned)gx, (unsigned)gy), per};
}

// src may alias dst exactly (test/unitest_mkl.cpp:33 calls MergeAddData(x, x, ...))
template <typename T>
__global__ void k_merge(const Cx<T>* src, Cx<T>* dst, T alpha, T beta, uint64_t num) {
    for (uint64_t i = gtid(); i < num; i += gstride()) dst[i] = merge_apply(src[i], dst[i], alpha, beta);
}

// Real parts of starts first..first+count-1 of a carousel run x [P][B][MN]
// (complex), gathered per start: dst [count][P][MN] -- the per-start output
// files of src/CPRA_MKL.cpp:186-209 (ComplexToReal, then each start's P planes).
template <typename T>
__global__ void k_real_starts(const Cx<T>* __restrict__ x, T* __restrict__ dst, uint64_t MN, uint64_t P, uint64_t B,
                              uint64_t first, uint64_t count) {
    const uint64_t total = count * P * MN;
    for (uint64_t e = gtid(); e < total; e += gstride()) {
        const uint64_t j = e % MN, plane = e / MN;
        dst[e] = x[((plane % P) * B + first + plane / P) * MN + j].x;
    }
}

// the same, four pixels per thread (MN % 4 == 0; x and dst 16-byte aligned):
// two 16-byte loads of (re, im, re, im), one 16-byte store of the reals
__global__ void k_real_starts4(const float4* __restrict__ x, float4* __restrict__ dst, uint64_t MN4, uint64_t P,
                               uint64_t B, uint64_t first, uint64_t count) {
    const uint64_t total = count * P * MN4;
    for (uint64_t e = gtid(); e < total; e += gstride()) {
        const uint64_t j = e % MN4, plane = e / MN4;
        const float4* s = x + 2 * (((plane % P) * B + first + plane / P) * MN4 + j);
        const float4 a = s[0], b = s[1];
        dst[e] = make_float4(a.x, a.z, b.x, b.z);
    }
}

template <typename T>
__global__ void k_scale(Cx<T>* __restrict__ x, T f, uint64_t num) {
    for (uint64_t i = gtid(); i < num; i += gstride()) x[i] = cscale(x[i], f);
}

// In-place fftshift of [batch][M][N] planes: element (r, c) trades places with
// ((r + M/2) % M, (c + N/2) % N), which is MKL_Impl.inl:180-209's quadrant swap
// for even sizes and a one-axis shift when one size is 1.  Each pair is
// visited once (from its member with r < M/2, or c < N/2 when M == 1).
template <typename T>
__global__ void k_shift2d(Cx<T>* __restrict__ x, uint64_t M, uint64_t N, uint64_t batch) {
    const uint64_t rows = (M >= 2) ? M / 2 : 1;
    const uint64_t cols = (M >= 2) ? N : N / 2;
    const uint64_t total = batch * rows * cols;
    for (uint64_t e = gtid(); e < total; e += gstride()) {
        const uint64_t c = e % cols;
        const uint64_t r = (e / cols) % rows;
        const uint64_t b = e / (cols * rows);
        const uint64_t r2 = (r + M / 2) % M, c2 = (c + N / 2) % N;
        Cx<T>* base = x + b * M * N;
        const Cx<T> u = base[r * N + c];
        base[r * N + c] = base[r2 * N + c2];
        base[r2 * N + c2] = u;
    }
}

// [batch][L][M][N] volumes: MKL_Impl.inl:212-251's octant swap
template <typename T>
__global__ void k_shift3d(Cx<T>* __restrict__ x, uint64_t M, uint64_t N, uint64_t L, uint64_t batch) {
    const uint64_t deps = (L >= 2) ? L / 2 : 1;
    const uint64_t rows = (L >= 2) ? M : ((M >= 2) ? M / 2 : 1);
    const uint64_t cols = (L >= 2 || M >= 2) ? N : N / 2;
    const uint64_t total = batch * deps * rows * cols;
    for (uint64_t e = gtid(); e < total; e += gstride()) {
        const uint64_t c = e % cols;
        const uint64_t r = (e / cols) % rows;
        const uint64_t d = (e / (cols * rows)) % deps;
        const uint64_t b = e / (cols * rows * deps);
        const uint64_t d2 = (d + L / 2) % L, r2 = (r + M / 2) % M, c2 = (c + N / 2) % N;
        Cx<T>* base = x + b * L * M * N;
        const uint64_t i1 = (d * M + r) * N + c, i2 = (d2 * M + r2) * N + c2;
        const Cx<T> u = base[i1];
        base[i1] = base[i2];
        base[i2] = u;
    }
}

// splitmix64 finaliser (S. Vigna), a counter-based stream: value i of stream
// (seed, id) depends only on (seed, id, i), not on the launch shape
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <typename T>
__global__ void k_uniform(T* __restrict__ x, uint64_t num, uint64_t key) {
    for (uint64_t i = gtid(); i < num; i += gstride()) {
        const uint64_t r = mix64(key + mix64(i));
        if constexpr (sizeof(T) == 4)
            x[i] = (float)(r >> 40) * 0x1.0p-24f;  // [0, 1), 24 random bits
        else
            x[i] = (double)(r >> 11) * 0x1.0p-53;  // [0, 1), 53 random bits
    }
}

// Sums of |a|^2 and |b|^2 over member i's `span` elements, in double.
// Stage 1: grid (CONVERGE_BLOCKS, batch); each block writes one partial pair.
template <typename T>
__global__ void k_norm_partial(const Cx<T>* __restrict__ a, const Cx<T>* __restrict__ b, uint64_t span,
                               uint64_t stride, double* __restrict__ partials) {
    __shared__ double sa[EW_THREADS], sb[EW_THREADS];
    const uint64_t m = blockIdx.y;
    const Cx<T>* pa = a + m * stride;
    const Cx<T>* pb = b + m * stride;
    double accA = 0.0, accB = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)EW_THREADS + threadIdx.x; i < span;
         i += (uint64_t)gridDim.x * EW_THREADS) {
        const Cx<T> u = pa[i], v = pb[i];
        accA = fma((double)u.x, (double)u.x, fma((double)u.y, (double)u.y, accA));
        accB = fma((double)v.x, (double)v.x, fma((double)v.y, (double)v.y, accB));
    }
    sa[threadIdx.x] = accA;
    sb[threadIdx.x] = accB;
    __syncthreads();
    for (int h = EW_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sa[threadIdx.x] += sa[threadIdx.x + h];
            sb[threadIdx.x] += sb[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[(m * gridDim.x + blockIdx.x) * 2 + 0] = sa[0];
        partials[(m * gridDim.x + blockIdx.x) * 2 + 1] = sb[0];
    }
}

// Stage 2: member i's partials summed in index order (deterministic)
__global__ void k_norm_final(const double* __restrict__ partials, double* __restrict__ sums, uint64_t batch,
                             int blocks) {
    for (uint64_t m = gtid(); m < batch; m += gstride()) {
        double sA = 0.0, sB = 0.0;
        for (int k = 0; k < blocks; ++k) {
            sA += partials[(m * blocks + k) * 2 + 0];
            sB += partials[(m * blocks + k) * 2 + 1];
        }
        sums[2 * m + 0] = sA;
        sums[2 * m + 1] = sB;
    }
}

// R-factor stage 1: grid (CONVERGE_BLOCKS, batch); |F| and the differences in
// double, one partial pair per block
template <typename T>
__global__ void k_rfactor_partial(const Cx<T>* __restrict__ F, const T* __restrict__ A, uint64_t a_stride,
                                  uint64_t plane, double* __restrict__ partials) {
    __shared__ double sd[EW_THREADS], sa[EW_THREADS];
    const uint64_t b = blockIdx.y;
    const Cx<T>* f = F + b * plane;
    const T* a = A + b * a_stride;
    double accD = 0.0, accA = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)EW_THREADS + threadIdx.x; i < plane;
         i += (uint64_t)gridDim.x * EW_THREADS) {
        const Cx<T> z = f[i];
        const double mag = sqrt(fma((double)z.x, (double)z.x, (double)z.y * (double)z.y));
        const double av = (double)a[i];
        accD += fabs(mag - av);
        accA += av;
    }
    sd[threadIdx.x] = accD;
    sa[threadIdx.x] = accA;
    __syncthreads();
    for (int h = EW_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sd[threadIdx.x] += sd[threadIdx.x + h];
            sa[threadIdx.x] += sa[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[(b * gridDim.x + blockIdx.x) * 2 + 0] = sd[0];
        partials[(b * gridDim.x + blockIdx.x) * 2 + 1] = sa[0];
    }
}

// C round(): halfway cases away from zero
__device__ __forceinline__ double round_away(double v) { return round(v); }

// Deterministic gather form of ker_Real2DTo3DInterpolation +
// ker_NormRealInterpolation (CUDA_Impl_Kernel.cuh:68-119).  Forward mapping of
// slice pixel (xIn, yIn) of slice p (column-major, yIn fastest): xr = xIn - N/2,
// yr = M/2 - yIn, 3D point (yr sin a, xr, yr cos a), nearest voxel (j, k, l)
// stored at z = L/2 - j, x = N/2 + k, y = M/2 - l, flat z*M*N + x*M + y, weight
// 50 for distance <= 0.02 else 1/distance, skipped for distance >= 0.5.  A
// voxel can only be reached from the pixel with xIn = x and yr the integer
// nearest to j sin a + l cos a (any other yr is >= 0.5 away along the slice),
// so each voxel visits every slice once and sums its weights in slice order.
template <typename T>
__global__ void k_real2d_to_3d(const T* __restrict__ src, T* __restrict__ dst, const T* __restrict__ ang,
                               int64_t M, int64_t N, int64_t P, int64_t L) {
    const uint64_t total = (uint64_t)M * N * L;
    for (uint64_t idx = gtid(); idx < total; idx += gstride()) {
        const int64_t y = (int64_t)(idx % M);
        const int64_t x = (int64_t)((idx / M) % N);
        const int64_t z = (int64_t)(idx / ((uint64_t)M * N));
        const int64_t j = L / 2 - z, l = M / 2 - y;
        double acc = 0.0, wsum = 0.0;
        for (int64_t p = 0; p < P; ++p) {
            const double a = (double)ang[p];
            const double sa = sin(a), ca = cos(a);
            const double yr = rint((double)j * sa + (double)l * ca);
            const int64_t yIn = M / 2 - (int64_t)yr;
            if (yIn < 0 || yIn >= M) continue;
            const double x3 = yr * sa, z3 = yr * ca;
            if ((int64_t)round_away(x3) != j || (int64_t)round_away(z3) != l) continue;
            const double dist = sqrt((x3 - (double)j) * (x3 - (double)j) + (z3 - (double)l) * (z3 - (double)l));
            if (!(dist < 0.5)) continue;
            const double w = (dist <= 0.02) ? 50.0 : 1.0 / dist;
            acc += w * (double)src[p * M * N + x * M + yIn];
            wsum += w;
        }
        dst[idx] = (wsum > 0.0) ? (T)(acc / wsum) : (T)0;
    }
}

// Complex2DTo3DInterpolation (the reference leaves it a stub,
// include/CUDA_Impl.cuh:89): gather-form trilinear merge of P complex central
// slices into a [L][N][M] volume with the geometry of the real merge above.
// Voxel (z, x, y) is the point (j, k, l) = (L/2 - z, x - N/2, M/2 - y); for
// slice p at angle a its in-plane coordinates are (yr, xr) = (j sin a + l cos
// a, k) and its distance to the plane is d = j cos a - l sin a.  Slices with
// |d| < 1 contribute (1 - |d|) times the slice linearly sampled at
// (yIn, xIn) = (M/2 - yr, N/2 + k); the voxel is the weight-normalised sum, or
// 0 (left unconstrained by the complex DataConstraint) when nothing reaches it.
// Coordinates, weights and sums are in the element type T, as the
// reference's merge kernel computes (CUDA_Impl_Kernel.cuh:68-108); the
// sines and cosines are evaluated once per slice in double and rounded to T.
// The part of one slice's contribution that depends only on the voxel's
// (j, l) and the slice: false if the plane is too far, else its weight wd,
// the first sampled row y0 and the fraction fy.
template <typename T>
__device__ __forceinline__ bool merge_plane(int64_t M, T j, T l, T sa, T ca, T& wd, int64_t& y0, T& fy) {
    const T d = j * ca - l * sa;
    wd = T(1) - (d < T(0) ? -d : d);
    if (!(wd > T(0))) return false;
    const T yIn = (T)(M / 2) - (j * sa + l * ca);
    const T y0f = floor(yIn);
    y0 = (int64_t)y0f;
    fy = yIn - y0f;
    return true;
}
// the rest for the voxel column x: the row of the slice at x (`row`, M
// pixels) sampled linearly at y0 + fy, weighted by wd into the sums
template <typename T>
__device__ __forceinline__ void merge_row(const Cx<T>* __restrict__ row, int64_t M, T wd, int64_t y0, T fy, T& accx,
                                          T& accy, T& wsum) {
    T sx = T(0), sy = T(0), sw = T(0);
    for (int dy = 0; dy < 2; ++dy) {
        const int64_t yy = y0 + dy;
        const T wy = dy ? fy : T(1) - fy;
        if (yy < 0 || yy >= M || wy == T(0)) continue;
        const Cx<T> v = row[yy];
        sx += wy * v.x;
        sy += wy * v.y;
        sw += wy;
    }
    if (sw == T(0)) return;
    accx += wd * sx;
    accy += wd * sy;
    wsum += wd * sw;
}
template <typename T>
__device__ __forceinline__ void merge_slice(const Cx<T>* __restrict__ src, int64_t p, int64_t M, int64_t N,
                                            int64_t x, T j, T l, T sa, T ca, T& accx, T& accy, T& wsum) {
    T wd, fy;
    int64_t y0;
    if (!merge_plane(M, j, l, sa, ca, wd, y0, fy)) return;
    merge_row(src + p * M * N + x * M, M, wd, y0, fy, accx, accy, wsum);
}

template <typename T>
struct SinCos2 {
    T s, c;
};

// every slice visited: the slices' sines and cosines staged per block in
// shared memory, MERGE_ANGLES at a time
constexpr int MERGE_ANGLES = 512;
template <typename T>
__global__ void __launch_bounds__(EW_THREADS) k_complex2d_to_3d(const Cx<T>* __restrict__ src, Cx<T>* __restrict__ dst,
                                                                const T* __restrict__ ang, int64_t M, int64_t N,
                                                                int64_t P, int64_t L) {
    __shared__ SinCos2<T> sc[MERGE_ANGLES];
    const uint64_t total = (uint64_t)M * N * L;
    const uint64_t iters = (total + gstride() - 1) / gstride();  // the same for every thread of the block
    for (uint64_t it = 0, idx = gtid(); it < iters; ++it, idx += gstride()) {
        const bool live = idx < total;
        const int64_t y = live ? (int64_t)(idx % M) : 0;
        const int64_t x = live ? (int64_t)((idx / M) % N) : 0;
        const int64_t z = live ? (int64_t)(idx / ((uint64_t)M * N)) : 0;
        const T j = (T)(L / 2 - z), l = (T)(M / 2 - y);
        T accx = T(0), accy = T(0), wsum = T(0);
        for (int64_t p0 = 0; p0 < P; p0 += MERGE_ANGLES) {
            const int64_t np = (P - p0 < MERGE_ANGLES) ? P - p0 : MERGE_ANGLES;
            __syncthreads();
            for (int64_t k = threadIdx.x; k < np; k += blockDim.x) {
                const double a = (double)ang[p0 + k];
                sc[k] = SinCos2<T>{(T)sin(a), (T)cos(a)};
            }
            __syncthreads();
            if (!live) continue;
            for (int64_t k = 0; k < np; ++k) merge_slice(src, p0 + k, M, N, x, j, l, sc[k].s, sc[k].c, accx, accy, wsum);
        }
        if (live) dst[idx] = (wsum > T(0)) ? Cx<T>{accx / wsum, accy / wsum} : Cx<T>{T(0), T(0)};
    }
}

// the same merge visiting only the slices that can reach the voxel
// (angle_table.cuh), in direction order; the work handed out dynamically.
// A work item is XC voxels along the tilt axis at one (z, y): the slices
// near them and each slice's plane terms depend only on (z, y), so they are
// found once for the item, and each voxel sums its slices in the same order
// as alone.  Consecutive items take consecutive y (coalesced rows and stores).
template <typename T, int XC>
__global__ void __launch_bounds__(EW_THREADS) k_complex2d_to_3d_w(const Cx<T>* __restrict__ src,
                                                                  Cx<T>* __restrict__ dst, const AngleTable tab,
                                                                  int64_t M, int64_t N, int64_t L) {
    const int64_t chunks = N / XC;
    const uint64_t total = (uint64_t)M * chunks * L;
    for_voxels_dynamic(tab.next, total, [&](uint64_t idx) {
        const int64_t y = (int64_t)(idx % M);
        const int64_t x0 = (int64_t)((idx / M) % chunks) * XC;
        const int64_t z = (int64_t)(idx / ((uint64_t)M * chunks));
        const T j = (T)(L / 2 - z), l = (T)(M / 2 - y);
        T accx[XC], accy[XC], wsum[XC];
#pragma unroll
        for (int t = 0; t < XC; ++t) accx[t] = accy[t] = wsum[t] = T(0);
        for_slices_near(tab, (double)(L / 2 - z), (double)(M / 2 - y), [&](int64_t p, double sa, double ca) {
            T wd, fy;
            int64_t y0;
            if (!merge_plane(M, j, l, (T)sa, (T)ca, wd, y0, fy)) return;
            const Cx<T>* __restrict__ rows = src + p * M * N + x0 * M;
#pragma unroll
            for (int t = 0; t < XC; ++t) merge_row(rows + t * M, M, wd, y0, fy, accx[t], accy[t], wsum[t]);
        });
#pragma unroll
        for (int t = 0; t < XC; ++t)
            dst[((uint64_t)z * N + x0 + t) * M + y] =
                (wsum[t] > T(0)) ? Cx<T>{accx[t] / wsum[t], accy[t] / wsum[t]} : Cx<T>{T(0), T(0)};
    });
}

// the windowed merge: four voxels per item where the side allows
template <typename T>
cudaError_t merge_windowed(const Cx<T>* src, Cx<T>* dst, const AngleTable& t, int64_t m, int64_t n, int64_t l,
                           cudaStream_t st) {
    if (n % 4 == 0)
        k_complex2d_to_3d_w<T, 4><<<resident_grid(k_complex2d_to_3d_w<T, 4>, EW_THREADS), EW_THREADS, 0, st>>>(
            src, dst, t, m, n, l);
    else
        k_complex2d_to_3d_w<T, 1><<<resident_grid(k_complex2d_to_3d_w<T, 1>, EW_THREADS), EW_THREADS, 0, st>>>(
            src, dst, t, m, n, l);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_space_constraint(bool dbl, void* x, const void* s, uint64_t num, uint64_t plane, int mode,
                                    cudaStream_t st) {
    const BroadcastGrid g = broadcast_grid(num, plane);
    if (dbl)
        k_space<double><<<g.grid, EW_THREADS, 0, st>>>((Cx<double>*)x, (const double*)s, num, plane, g.reps_per_y,
                                                       mode);
    else
        k_space<float><<<g.grid, EW_THREADS, 0, st>>>((Cx<float>*)x, (const float*)s, num, plane, g.reps_per_y, mode);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_data_constraint_real(bool dbl, void* x, const void* a, uint64_t num, uint64_t plane, int mode,
                                        cudaStream_t st) {
    const BroadcastGrid g = broadcast_grid(num, plane);
    if (dbl)
        k_data_real<double><<<g.grid, EW_THREADS, 0, st>>>((Cx<double>*)x, (const double*)a, num, plane,
                                                           g.reps_per_y, mode);
    else
        k_data_real<float><<<g.grid, EW_THREADS, 0, st>>>((Cx<float>*)x, (const float*)a, num, plane, g.reps_per_y,
                                                          mode);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_data_constraint_complex(bool dbl, void* x, const void* c, uint64_t num, uint64_t plane,
                                           cudaStream_t st) {
    const BroadcastGrid g = broadcast_grid(num, plane);
    if (dbl)
        k_data_complex<double><<<g.grid, EW_THREADS, 0, st>>>((Cx<double>*)x, (const Cx<double>*)c, num, plane,
                                                              g.reps_per_y);
    else
        k_data_complex<float><<<g.grid, EW_THREADS, 0, st>>>((Cx<float>*)x, (const Cx<float>*)c, num, plane,
                                                             g.reps_per_y);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_merge_add(bool dbl, const void* src, void* dst, double alpha, double beta, uint64_t num,
                             cudaStream_t st) {
    const unsigned g = ew_grid(num, EW_THREADS);
    if (dbl)
        k_merge<double><<<g, EW_THREADS, 0, st>>>((const Cx<double>*)src, (Cx<double>*)dst, alpha, beta, num);
    else
        k_merge<float><<<g, EW_THREADS, 0, st>>>((const Cx<float>*)src, (Cx<float>*)dst, (float)alpha,
                                                 (float)beta, num);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_real_starts(bool dbl, const void* x, void* dst, uint64_t MN, uint64_t P, uint64_t B, uint64_t first,
                               uint64_t count, cudaStream_t st) {
    const uint64_t total = count * P * MN;
    if (total == 0) return cudaSuccess;
    const bool vec = !dbl && MN % 4 == 0 && (reinterpret_cast<uintptr_t>(x) & 15u) == 0 &&
                     (reinterpret_cast<uintptr_t>(dst) & 15u) == 0;
    if (vec)
        k_real_starts4<<<ew_grid(total / 4, EW_THREADS), EW_THREADS, 0, st>>>((const float4*)x, (float4*)dst, MN / 4,
                                                                             P, B, first, count);
    else if (dbl)
        k_real_starts<double><<<ew_grid(total, EW_THREADS), EW_THREADS, 0, st>>>((const Cx<double>*)x, (double*)dst,
                                                                                MN, P, B, first, count);
    else
        k_real_starts<float><<<ew_grid(total, EW_THREADS), EW_THREADS, 0, st>>>((const Cx<float>*)x, (float*)dst, MN,
                                                                               P, B, first, count);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_scale(bool dbl, void* x, double factor, uint64_t num, cudaStream_t st) {
    const unsigned g = ew_grid(num, EW_THREADS);
    if (dbl)
        k_scale<double><<<g, EW_THREADS, 0, st>>>((Cx<double>*)x, factor, num);
    else
        k_scale<float><<<g, EW_THREADS, 0, st>>>((Cx<float>*)x, (float)factor, num);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_fftshift2d(bool dbl, void* x, uint64_t M, uint64_t N, uint64_t batch, cudaStream_t st) {
    const uint64_t work = batch * M * N / 2;
    if (work == 0) return cudaSuccess;
    const unsigned g = ew_grid(work, EW_THREADS);
    if (dbl)
        k_shift2d<double><<<g, EW_THREADS, 0, st>>>((Cx<double>*)x, M, N, batch);
    else
        k_shift2d<float><<<g, EW_THREADS, 0, st>>>((Cx<float>*)x, M, N, batch);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_fftshift3d(bool dbl, void* x, uint64_t M, uint64_t N, uint64_t L, uint64_t batch,
                              cudaStream_t st) {
    const uint64_t work = batch * M * N * L / 2;
    if (work == 0) return cudaSuccess;
    const unsigned g = ew_grid(work, EW_THREADS);
    if (dbl)
        k_shift3d<double><<<g, EW_THREADS, 0, st>>>((Cx<double>*)x, M, N, L, batch);
    else
        k_shift3d<float><<<g, EW_THREADS, 0, st>>>((Cx<float>*)x, M, N, L, batch);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_uniform(bool dbl, void* x, uint64_t num, uint64_t seed, uint64_t stream_id, cudaStream_t st) {
    const unsigned g = ew_grid(num, EW_THREADS);
    const uint64_t key = seed * 0xD1B54A32D192ED03ull + stream_id * 0x8CB92BA72F3D8DD7ull;
    if (dbl)
        k_uniform<double><<<g, EW_THREADS, 0, st>>>((double*)x, num, key);
    else
        k_uniform<float><<<g, EW_THREADS, 0, st>>>((float*)x, num, key);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_norm_pairs(bool dbl, const void* a, const void* b, uint64_t span, uint64_t stride,
                              uint64_t batch, double* partials, double* sums, cudaStream_t st) {
    if (batch == 0) return cudaSuccess;
    if (batch > 65535) return cudaErrorInvalidValue;
    dim3 grid(CONVERGE_BLOCKS, (unsigned)batch);
    if (dbl)
        k_norm_partial<double><<<grid, EW_THREADS, 0, st>>>((const Cx<double>*)a, (const Cx<double>*)b, span,
                                                            stride, partials);
    else
        k_norm_partial<float><<<grid, EW_THREADS, 0, st>>>((const Cx<float>*)a, (const Cx<float>*)b, span, stride,
                                                           partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_norm_final<<<ew_grid(batch, 64), 64, 0, st>>>(partials, sums, batch, CONVERGE_BLOCKS);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_norm_final(const double* partials, double* sums, uint64_t batch, cudaStream_t st) {
    k_norm_final<<<ew_grid(batch, 64), 64, 0, st>>>(partials, sums, batch, CONVERGE_BLOCKS);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_rfactor_sums(bool dbl, const void* F, const void* A, uint64_t a_stride, uint64_t plane,
                                uint64_t batch, double* partials, double* sums, cudaStream_t st) {
    if (batch == 0) return cudaSuccess;
    if (batch > 65535) return cudaErrorInvalidValue;
    dim3 grid(CONVERGE_BLOCKS, (unsigned)batch);
    if (dbl)
        k_rfactor_partial<double><<<grid, EW_THREADS, 0, st>>>((const Cx<double>*)F, (const double*)A, a_stride, plane,
                                                               partials);
    else
        k_rfactor_partial<float><<<grid, EW_THREADS, 0, st>>>((const Cx<float>*)F, (const float*)A, a_stride, plane,
                                                              partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_norm_final<<<ew_grid(batch, 64), 64, 0, st>>>(partials, sums, batch, CONVERGE_BLOCKS);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_real2d_to_3d(bool dbl, const void* src, void* dst, const void* angles, uint64_t m, uint64_t n,
                                uint64_t p, uint64_t l, cudaStream_t st) {
    const uint64_t total = m * n * l;
    if (total == 0) return cudaSuccess;
    const unsigned g = ew_grid(total, EW_THREADS);
    if (dbl)
        k_real2d_to_3d<double><<<g, EW_THREADS, 0, st>>>((const double*)src, (double*)dst, (const double*)angles,
                                                         (int64_t)m, (int64_t)n, (int64_t)p, (int64_t)l);
    else
        k_real2d_to_3d<float><<<g, EW_THREADS, 0, st>>>((const float*)src, (float*)dst, (const float*)angles,
                                                        (int64_t)m, (int64_t)n, (int64_t)p, (int64_t)l);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_complex2d_to_3d(bool dbl, const void* src, void* dst, const void* angles, uint64_t m,
                                   uint64_t n, uint64_t p, uint64_t l, void* atab, cudaStream_t st) {
    const uint64_t total = m * n * l;
    if (total == 0) return cudaSuccess;
    const unsigned g = ew_grid(total, EW_THREADS);
    if (atab && p <= (uint64_t)ANGLE_TABLE_MAX) {
        cudaError_t e = dbl ? launch_sort_angles<double>((const double*)angles, (int64_t)p, atab, st)
                            : launch_sort_angles<float>((const float*)angles, (int64_t)p, atab, st);
        if (e != cudaSuccess) return e;
        const AngleTable t = angle_table_view(atab, (int64_t)p);
        e = cudaMemsetAsync(t.next, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
        e = dbl ? merge_windowed<double>((const Cx<double>*)src, (Cx<double>*)dst, t, (int64_t)m, (int64_t)n,
                                         (int64_t)l, st)
                : merge_windowed<float>((const Cx<float>*)src, (Cx<float>*)dst, t, (int64_t)m, (int64_t)n,
                                        (int64_t)l, st);
        count_launches(2);
        return e;
    }
    if (dbl)
        k_complex2d_to_3d<double><<<g, EW_THREADS, 0, st>>>((const Cx<double>*)src, (Cx<double>*)dst,
                                                            (const double*)angles, (int64_t)m, (int64_t)n,
                                                            (int64_t)p, (int64_t)l);
    else
        k_complex2d_to_3d<float><<<g, EW_THREADS, 0, st>>>((const Cx<float>*)src, (Cx<float>*)dst,
                                                           (const float*)angles, (int64_t)m, (int64_t)n,
                                                           (int64_t)p, (int64_t)l);
    count_launches();
    return cudaGetLastError();
}

}  // namespace cpra_b200
