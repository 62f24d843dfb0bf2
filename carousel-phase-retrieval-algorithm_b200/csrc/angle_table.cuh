// Slices ordered by their line direction, for gathers over the slices per
// voxel (the merge's geometry: slice p's points in the (z, y) plane of the
// volume lie on the line through the centre with direction (sin a_p, cos a_p)).
// A voxel at polar angle phi = atan2(cz, cy) and distance rho from the tilt
// axis can receive a contribution of slice p only if its distance to that
// line, rho |sin(phi - a_p)|, is below sqrt(2) (both bilinear weights
// positive), so only slices with a_p within asin(1.5 / rho) of phi (mod pi)
// are visited; near the axis (rho <= 1.5) all are.
//
// The table: the P directions a_p mod pi sorted ascending (ties by p), their
// slice indices, and sin a_p, cos a_p; built by one block per call
// (k_sort_angles, a bitonic sort in shared memory, deterministic).
#pragma once
#include <cstdint>

#include "cpra_common.cuh"

namespace cpra_b200 {

constexpr int ANGLE_TABLE_MAX = 4096;  // slices; above this the gathers visit every slice
constexpr double ANGLE_PI = 3.141592653589793238462643383279502884;

struct AngleTable {
    const double* key;  // [P] direction mod pi, ascending
    const int* idx;     // [P] slice index
    const double2* sc;  // [P] (sin a, cos a) of that slice
    int64_t P;
    unsigned long long* next;  // work counter of the gather that reads the table (zeroed before its launch)
};

// byte offsets of the three arrays in a table buffer of angle_table_bytes(P)
__host__ __device__ inline uint64_t angle_table_idx_offset(uint64_t P) { return (P * 8 + 255) / 256 * 256; }
__host__ __device__ inline uint64_t angle_table_sc_offset(uint64_t P) {
    return angle_table_idx_offset(P) + (P * 4 + 255) / 256 * 256;
}
__host__ __device__ inline uint64_t angle_table_next_offset(uint64_t P) {
    return angle_table_sc_offset(P) + (P * 16 + 255) / 256 * 256;
}
__host__ __device__ inline uint64_t angle_table_bytes(uint64_t P) { return angle_table_next_offset(P) + 256; }

inline AngleTable angle_table_view(void* buf, int64_t P) {
    char* b = static_cast<char*>(buf);
    return AngleTable{reinterpret_cast<const double*>(b), reinterpret_cast<const int*>(b + angle_table_idx_offset(P)),
                      reinterpret_cast<const double2*>(b + angle_table_sc_offset(P)), P,
                      reinterpret_cast<unsigned long long*>(b + angle_table_next_offset(P))};
}

// The voxels of a gather over slices cost very different amounts (a voxel
// near the tilt axis is near many slices, a far one near few), so the work
// items (voxels, or short runs of them) are handed out dynamically: each warp
// takes 32 * GATHER_VOXELS_PER_LANE consecutive item indices from the
// counter at a time until all `total` are done, and calls f(i) for each of
// its lanes' indices.  Every item is still computed by one thread with the
// same arithmetic.  Launch exactly the resident CTAs (the counter replaces
// the grid-stride loop) with the counter zeroed on the same stream; all 32
// lanes of every warp take part.
constexpr int GATHER_VOXELS_PER_LANE = 4;
template <class Fn>
__device__ __forceinline__ void for_voxels_dynamic(unsigned long long* next, uint64_t total, Fn f) {
    const int lane = threadIdx.x & 31;
    constexpr unsigned long long CHUNK = 32ull * GATHER_VOXELS_PER_LANE;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(next, CHUNK);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) return;
#pragma unroll 1
        for (int r = 0; r < GATHER_VOXELS_PER_LANE; ++r) {
            const uint64_t i = base + (uint64_t)r * 32 + (uint64_t)lane;
            if (i < total) f(i);
        }
    }
}

// CTAs of `kernel` resident on the whole device at `threads` per CTA
template <class K>
inline unsigned resident_grid(K kernel, unsigned threads, size_t smem = 0) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, (int)threads, smem) != cudaSuccess || n < 1) {
        (void)cudaGetLastError();
        n = 1;
    }
    return (unsigned)n * (unsigned)sm_count();
}

// one block of 1024 threads; dynamic shared memory 12 * N bytes, N the
// power of two >= P (<= ANGLE_TABLE_MAX)
template <typename T>
__global__ void __launch_bounds__(1024) k_sort_angles(const T* __restrict__ ang, int64_t P, int N, double* key,
                                                      int* idx, double2* sc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sk = reinterpret_cast<double*>(smem_raw);
    int* si = reinterpret_cast<int*>(sk + N);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        if (i < P) {
            double k = fmod((double)ang[i], ANGLE_PI);
            if (k < 0.0) k += ANGLE_PI;
            if (k >= ANGLE_PI) k -= ANGLE_PI;
            sk[i] = k;
            si[i] = i;
        } else {
            sk[i] = 1e300;
            si[i] = 0x7fffffff;
        }
    }
    __syncthreads();
    // bitonic sort, ascending by (key, index)
    for (int k = 2; k <= N; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < N; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const bool gt = sk[i] > sk[l] || (sk[i] == sk[l] && si[i] > si[l]);
                    if (gt == up) {
                        const double tk = sk[i];
                        sk[i] = sk[l];
                        sk[l] = tk;
                        const int ti = si[i];
                        si[i] = si[l];
                        si[l] = ti;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        key[i] = sk[i];
        idx[i] = si[i];
        const double a = (double)ang[si[i]];
        sc[i] = make_double2(sin(a), cos(a));
    }
}

template <typename T>
cudaError_t launch_sort_angles(const T* ang, int64_t P, void* buf, cudaStream_t st) {
    int N = 1;
    while (N < P) N <<= 1;
    char* b = static_cast<char*>(buf);
    const size_t smem = (size_t)N * 12;
    cudaError_t e = cudaFuncSetAttribute(k_sort_angles<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_sort_angles<T><<<1, 1024, smem, st>>>(ang, P, N, reinterpret_cast<double*>(b),
                                             reinterpret_cast<int*>(b + angle_table_idx_offset(P)),
                                             reinterpret_cast<double2*>(b + angle_table_sc_offset(P)));
    return cudaGetLastError();
}

// first k with key[k] >= a
__device__ __forceinline__ int64_t angle_lower_bound(const double* key, int64_t P, double a) {
    int64_t lo = 0, hi = P;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (key[mid] < a)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// f(p, sin a_p, cos a_p) for the slices that can reach the voxel at (cz, cy)
// (cz = L/2 - z, cy = M/2 - y), in ascending direction order.  The window
// only prunes (the caller's weights decide), so it is computed in float and
// widened by 1e-4 rad, far above the float rounding of its bounds.
template <class Fn>
__device__ __forceinline__ void for_slices_near(const AngleTable& t, double cz, double cy, Fn f) {
    const float czf = (float)cz, cyf = (float)cy;
    const float rho = sqrtf(czf * czf + cyf * cyf);
    auto range = [&](double a, double b) {
        for (int64_t k = angle_lower_bound(t.key, t.P, a); k < t.P && t.key[k] <= b; ++k) {
            const double2 w = t.sc[k];
            f((int64_t)t.idx[k], w.x, w.y);
        }
    };
    if (!(rho > 1.51f)) {
        range(-1.0, 4.0);
        return;
    }
    const double delta0 = (double)asinf(1.5f / rho);
    if (delta0 >= 0.5 * ANGLE_PI - 1e-3) {  // the two windows would meet
        range(-1.0, 4.0);
        return;
    }
    double phi = (double)atan2f(czf, cyf);
    if (phi < 0.0) phi += ANGLE_PI;
    if (phi >= ANGLE_PI) phi -= ANGLE_PI;
    const double delta = delta0 + 1e-4;
    const double lo = phi - delta, hi = phi + delta;
    if (lo < 0.0) {
        range(-1.0, hi);
        range(lo + ANGLE_PI, 4.0);
    } else if (hi >= ANGLE_PI) {
        range(lo, 4.0);
        range(-1.0, hi - ANGLE_PI);
    } else {
        range(lo, hi);
    }
}

}  // namespace cpra_b200
