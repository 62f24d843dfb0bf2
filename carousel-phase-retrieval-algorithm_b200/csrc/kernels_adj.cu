// Central slices of a 3D Fourier volume and the adjoints of the amplitude loss
// (project-defined; the reference has no slice operator, loss or gradient).
//
// Geometry: the merges' (CUDA_Impl_Kernel.cuh:80-90).  A volume is [L][N][M]
// (y fastest); voxel (z, x, y) sits at the point (j, k, l) = (L/2 - z,
// x - N/2, M/2 - y).  Slice pixel (xIn, yIn) of angle a, slices stored
// [P][N][M] (yIn fastest), is the point (yr sin a, xr, yr cos a) with
// xr = xIn - N/2, yr = M/2 - yIn, i.e. the voxel coordinates
//   z = L/2 - yr sin a,  x = xIn,  y = M/2 - yr cos a.
// The x coordinate is integral, so trilinear interpolation reduces to
// bilinear interpolation in (z, y) on the plane x = xIn:
//   s[p](xIn, yIn) = sum_{z,y} w(z) w(y) V[z][xIn][y],  w(u) = max(0, 1 - |u - u*|)
// (points outside the volume contribute 0).
//
// Loss L = sum_p sum_px (|s| - A)^2 with G = 2 (|s| - A) s / |s| (0 where s = 0),
// the derivative with respect to Re s + i Im s:
//   dL/dV (Re + i Im)  = S^T G: each voxel gathers w * G from the pixels whose
//                        bilinear footprint covers it (at most 3 rows per slice,
//                        found from the voxel), so the sum is deterministic;
//   dL/da_p            = sum_px Re(conj(G) ds/da), ds/da from the derivative of
//                        the weights (dz/da = -yr cos a, dy/da = yr sin a).
// Coordinates and weights are computed in double; data stay in T.
#include "cpra_internal.h"
#include "ops_ew.cuh"

namespace cpra_b200 {
namespace {

constexpr int ADJ_THREADS = 256;

__device__ __forceinline__ uint64_t tid_g() { return blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t str_g() { return (uint64_t)gridDim.x * blockDim.x; }

// slice value at pixel (p, xIn, yIn) and, optionally, its derivative in the angle
template <typename T>
__device__ __forceinline__ void sample(const Cx<T>* __restrict__ V, int64_t M, int64_t N, int64_t L, double sa,
                                       double ca, int64_t xIn, int64_t yIn, double& re, double& im, double* dre,
                                       double* dim) {
    const double yr = (double)(M / 2 - yIn);
    const double zf = (double)(L / 2) - yr * sa;
    const double yf = (double)(M / 2) - yr * ca;
    const double dz = -yr * ca, dy = yr * sa;  // dzf/da, dyf/da
    const int64_t z0 = (int64_t)floor(zf), y0 = (int64_t)floor(yf);
    const double fz = zf - (double)z0, fy = yf - (double)y0;
    re = im = 0.0;
    if (dre) *dre = *dim = 0.0;
    for (int a = 0; a < 2; ++a) {
        const int64_t z = z0 + a;
        if (z < 0 || z >= L) continue;
        const double wz = a ? fz : 1.0 - fz;
        const double dwz = a ? dz : -dz;  // d wz / d angle
        for (int b = 0; b < 2; ++b) {
            const int64_t y = y0 + b;
            if (y < 0 || y >= M) continue;
            const double wy = b ? fy : 1.0 - fy;
            const double dwy = b ? dy : -dy;
            const Cx<T> v = V[(z * N + xIn) * M + y];
            const double w = wz * wy;
            re += w * (double)v.x;
            im += w * (double)v.y;
            if (dre) {
                const double dw = dwz * wy + wz * dwy;
                *dre += dw * (double)v.x;
                *dim += dw * (double)v.y;
            }
        }
    }
}

template <typename T>
__global__ void k_slice(const Cx<T>* __restrict__ V, const T* __restrict__ ang, Cx<T>* __restrict__ out, int64_t M,
                        int64_t N, int64_t P, int64_t L) {
    const uint64_t total = (uint64_t)P * N * M;
    for (uint64_t i = tid_g(); i < total; i += str_g()) {
        const int64_t yIn = (int64_t)(i % M), xIn = (int64_t)((i / M) % N), p = (int64_t)(i / ((uint64_t)M * N));
        const double a = (double)ang[p];
        double re, im;
        sample(V, M, N, L, sin(a), cos(a), xIn, yIn, re, im, (double*)nullptr, (double*)nullptr);
        out[i] = Cx<T>{(T)re, (T)im};
    }
}

// G and the per-slice sums of the loss and of Re(conj(G) ds/da); grid
// (CONVERGE_BLOCKS, P), one partial pair per block
template <typename T>
__global__ void k_slice_residual(const Cx<T>* __restrict__ V, const T* __restrict__ ang, const T* __restrict__ A,
                                 Cx<T>* __restrict__ G, int64_t M, int64_t N, int64_t L, double* __restrict__ partials) {
    __shared__ double sl[ADJ_THREADS], sg[ADJ_THREADS];
    const int64_t p = blockIdx.y;
    const double a = (double)ang[p];
    const double sa = sin(a), ca = cos(a);
    const uint64_t plane = (uint64_t)N * M;
    double accL = 0.0, accT = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)ADJ_THREADS + threadIdx.x; i < plane; i += (uint64_t)gridDim.x * ADJ_THREADS) {
        const int64_t yIn = (int64_t)(i % M), xIn = (int64_t)(i / M);
        double re, im, dre, dim;
        sample(V, M, N, L, sa, ca, xIn, yIn, re, im, &dre, &dim);
        const double mag = sqrt(re * re + im * im);
        const double d = mag - (double)A[p * plane + i];
        accL += d * d;
        double gr = 0.0, gi = 0.0;
        if (mag > 0.0) {
            gr = 2.0 * d * re / mag;
            gi = 2.0 * d * im / mag;
        }
        G[p * plane + i] = Cx<T>{(T)gr, (T)gi};
        accT += gr * dre + gi * dim;
    }
    sl[threadIdx.x] = accL;
    sg[threadIdx.x] = accT;
    __syncthreads();
    for (int h = ADJ_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sl[threadIdx.x] += sl[threadIdx.x + h];
            sg[threadIdx.x] += sg[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[(p * gridDim.x + blockIdx.x) * 2 + 0] = sl[0];
        partials[(p * gridDim.x + blockIdx.x) * 2 + 1] = sg[0];
    }
}

// gradient with respect to V: each voxel gathers w * G over the slices
template <typename T>
__global__ void k_slice_adjoint(const Cx<T>* __restrict__ G, const T* __restrict__ ang, Cx<T>* __restrict__ gV,
                                int64_t M, int64_t N, int64_t P, int64_t L) {
    const uint64_t total = (uint64_t)L * N * M;
    for (uint64_t i = tid_g(); i < total; i += str_g()) {
        const int64_t y = (int64_t)(i % M), x = (int64_t)((i / M) % N), z = (int64_t)(i / ((uint64_t)M * N));
        double re = 0.0, im = 0.0;
        for (int64_t p = 0; p < P; ++p) {
            const double a = (double)ang[p];
            const double sa = sin(a), ca = cos(a);
            // rows whose point (zf, yf) = (L/2 - yr sa, M/2 - yr ca) lies within 1 of (z, y) in both axes
            double lo = -1e300, hi = 1e300;
            const double cz = (double)(L / 2) - (double)z, cy = (double)(M / 2) - (double)y;
            if (fabs(sa) > 1e-12) {
                const double r0 = (cz - 1.0) / sa, r1 = (cz + 1.0) / sa;
                lo = fmax(lo, fmin(r0, r1));
                hi = fmin(hi, fmax(r0, r1));
            } else if (fabs(cz) >= 1.0) {
                continue;
            }
            if (fabs(ca) > 1e-12) {
                const double r0 = (cy - 1.0) / ca, r1 = (cy + 1.0) / ca;
                lo = fmax(lo, fmin(r0, r1));
                hi = fmin(hi, fmax(r0, r1));
            } else if (fabs(cy) >= 1.0) {
                continue;
            }
            for (int64_t yr = (int64_t)ceil(lo); (double)yr <= hi; ++yr) {
                const int64_t yIn = M / 2 - yr;
                if (yIn < 0 || yIn >= M) continue;
                const double wz = 1.0 - fabs((double)(L / 2) - (double)yr * sa - (double)z);
                const double wy = 1.0 - fabs((double)(M / 2) - (double)yr * ca - (double)y);
                if (!(wz > 0.0) || !(wy > 0.0)) continue;
                const Cx<T> g = G[(p * N + x) * M + yIn];
                const double w = wz * wy;
                re += w * (double)g.x;
                im += w * (double)g.y;
            }
        }
        gV[i] = Cx<T>{(T)re, (T)im};
    }
}

}  // namespace

cudaError_t launch_slice(bool dbl, const void* V, const void* ang, void* out, uint64_t m, uint64_t n, uint64_t p,
                         uint64_t l, cudaStream_t st) {
    const uint64_t total = p * n * m;
    if (total == 0) return cudaSuccess;
    const unsigned g = ew_grid(total, ADJ_THREADS);
    if (dbl)
        k_slice<double><<<g, ADJ_THREADS, 0, st>>>((const Cx<double>*)V, (const double*)ang, (Cx<double>*)out, m, n,
                                                   p, l);
    else
        k_slice<float><<<g, ADJ_THREADS, 0, st>>>((const Cx<float>*)V, (const float*)ang, (Cx<float>*)out, m, n, p, l);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_slice_loss_grad(bool dbl, const void* V, const void* ang, const void* A, void* G, void* gV,
                                   uint64_t m, uint64_t n, uint64_t p, uint64_t l, double* partials, double* sums,
                                   cudaStream_t st) {
    if (p == 0) return cudaSuccess;
    if (p > 65535) return cudaErrorInvalidValue;
    dim3 grid(CONVERGE_BLOCKS, (unsigned)p);
    if (dbl)
        k_slice_residual<double><<<grid, ADJ_THREADS, 0, st>>>((const Cx<double>*)V, (const double*)ang,
                                                               (const double*)A, (Cx<double>*)G, m, n, l, partials);
    else
        k_slice_residual<float><<<grid, ADJ_THREADS, 0, st>>>((const Cx<float>*)V, (const float*)ang,
                                                              (const float*)A, (Cx<float>*)G, m, n, l, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = launch_norm_final(partials, sums, p, st);
    if (e != cudaSuccess) return e;
    const uint64_t vox = l * n * m;
    const unsigned g = ew_grid(vox, ADJ_THREADS);
    if (dbl)
        k_slice_adjoint<double><<<g, ADJ_THREADS, 0, st>>>((const Cx<double>*)G, (const double*)ang, (Cx<double>*)gV,
                                                           m, n, p, l);
    else
        k_slice_adjoint<float><<<g, ADJ_THREADS, 0, st>>>((const Cx<float>*)G, (const float*)ang, (Cx<float>*)gV, m,
                                                          n, p, l);
    count_launches(2);
    return cudaGetLastError();
}

}  // namespace cpra_b200
