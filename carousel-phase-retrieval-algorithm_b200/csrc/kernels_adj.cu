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
#include "angle_table.cuh"

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

// gradient with respect to V: each voxel gathers w * G over the slices.  The
// slices' sines, cosines and the reciprocals that bound each slice's rows are
// staged per block in shared memory, ADJ_ANGLES at a time, so the voxel loop
// evaluates no transcendental and no division.  The row window is computed in
// float and widened by 0.01 of a row: it only bounds the loop (rows are
// integers; its float rounding is below 1e-3 of a row at these coordinates),
// and the double weights decide which rows contribute, exactly as before.
constexpr int ADJ_ANGLES = 512;
struct AngleRow {
    double sa, ca;   // sin, cos
    float isa, ica;  // 1/sin (0 when |sin| <= 1e-12), 1/cos (likewise)
};

template <typename T>
__global__ void __launch_bounds__(ADJ_THREADS) k_slice_adjoint(const Cx<T>* __restrict__ G, const T* __restrict__ ang,
                                                               Cx<T>* __restrict__ gV, int64_t M, int64_t N,
                                                               int64_t P, int64_t L) {
    __shared__ AngleRow tab[ADJ_ANGLES];
    const uint64_t total = (uint64_t)L * N * M;
    // every thread of the block runs the same number of outer iterations
    const uint64_t iters = (total + str_g() - 1) / str_g();
    for (uint64_t it = 0, i = tid_g(); it < iters; ++it, i += str_g()) {
        const bool live = i < total;
        const int64_t y = live ? (int64_t)(i % M) : 0, x = live ? (int64_t)((i / M) % N) : 0;
        const int64_t z = live ? (int64_t)(i / ((uint64_t)M * N)) : 0;
        const float czf = (float)(L / 2 - z), cyf = (float)(M / 2 - y);
        double re = 0.0, im = 0.0;
        for (int64_t p0 = 0; p0 < P; p0 += ADJ_ANGLES) {
            const int64_t np = (P - p0 < ADJ_ANGLES) ? P - p0 : ADJ_ANGLES;
            __syncthreads();
            for (int64_t k = threadIdx.x; k < np; k += ADJ_THREADS) {
                const double a = (double)ang[p0 + k];
                const double sa = sin(a), ca = cos(a);
                tab[k] = AngleRow{sa, ca, fabs(sa) > 1e-12 ? (float)(1.0 / sa) : 0.0f,
                                  fabs(ca) > 1e-12 ? (float)(1.0 / ca) : 0.0f};
            }
            __syncthreads();
            if (!live) continue;
            for (int64_t k = 0; k < np; ++k) {
                const AngleRow w = tab[k];
                // rows whose point (zf, yf) = (L/2 - yr sa, M/2 - yr ca) lies within 1 of (z, y) in both axes
                float lo = -3.0e38f, hi = 3.0e38f;
                if (w.isa != 0.0f) {
                    const float r0 = (czf - 1.0f) * w.isa, r1 = (czf + 1.0f) * w.isa;
                    lo = fmaxf(lo, fminf(r0, r1));
                    hi = fminf(hi, fmaxf(r0, r1));
                } else if (fabsf(czf) >= 1.0f) {
                    continue;
                }
                if (w.ica != 0.0f) {
                    const float r0 = (cyf - 1.0f) * w.ica, r1 = (cyf + 1.0f) * w.ica;
                    lo = fmaxf(lo, fminf(r0, r1));
                    hi = fminf(hi, fmaxf(r0, r1));
                } else if (fabsf(cyf) >= 1.0f) {
                    continue;
                }
                if (lo > hi + 0.02f) continue;
                lo = fmaxf(lo, (float)(-M));  // rows outside the slice never contribute
                hi = fminf(hi, (float)M);
                const int64_t p = p0 + k;
                for (int64_t yr = (int64_t)ceilf(lo - 0.01f); (float)yr <= hi + 0.01f; ++yr) {
                    const int64_t yIn = M / 2 - yr;
                    if (yIn < 0 || yIn >= M) continue;
                    const double wz = 1.0 - fabs((double)(L / 2) - (double)yr * w.sa - (double)z);
                    const double wy = 1.0 - fabs((double)(M / 2) - (double)yr * w.ca - (double)y);
                    if (!(wz > 0.0) || !(wy > 0.0)) continue;
                    const Cx<T> g = G[(p * N + x) * M + yIn];
                    const double wt = wz * wy;
                    re += wt * (double)g.x;
                    im += wt * (double)g.y;
                }
            }
        }
        if (live) gV[i] = Cx<T>{(T)re, (T)im};
    }
}

// the same gather visiting only the slices that can reach the voxel
// (angle_table.cuh), in direction order; rows and weights as above, in double
template <typename T>
__global__ void __launch_bounds__(ADJ_THREADS) k_slice_adjoint_w(const Cx<T>* __restrict__ G, const AngleTable tab,
                                                                 Cx<T>* __restrict__ gV, int64_t M, int64_t N,
                                                                 int64_t L) {
    const uint64_t total = (uint64_t)L * N * M;
    for (uint64_t i = tid_g(); i < total; i += str_g()) {
        const int64_t y = (int64_t)(i % M), x = (int64_t)((i / M) % N), z = (int64_t)(i / ((uint64_t)M * N));
        const double cz = (double)(L / 2) - (double)z, cy = (double)(M / 2) - (double)y;
        double re = 0.0, im = 0.0;
        for_slices_near(tab, cz, cy, [&](int64_t p, double sa, double ca) {
            double lo = -1e300, hi = 1e300;
            if (fabs(sa) > 1e-12) {
                const double r0 = (cz - 1.0) / sa, r1 = (cz + 1.0) / sa;
                lo = fmax(lo, fmin(r0, r1));
                hi = fmin(hi, fmax(r0, r1));
            } else if (fabs(cz) >= 1.0) {
                return;
            }
            if (fabs(ca) > 1e-12) {
                const double r0 = (cy - 1.0) / ca, r1 = (cy + 1.0) / ca;
                lo = fmax(lo, fmin(r0, r1));
                hi = fmin(hi, fmax(r0, r1));
            } else if (fabs(cy) >= 1.0) {
                return;
            }
            lo = fmax(lo, (double)(-M));
            hi = fmin(hi, (double)M);
            for (int64_t yr = (int64_t)ceil(lo - 1e-9); (double)yr <= hi + 1e-9; ++yr) {
                const int64_t yIn = M / 2 - yr;
                if (yIn < 0 || yIn >= M) continue;
                const double wz = 1.0 - fabs((double)(L / 2) - (double)yr * sa - (double)z);
                const double wy = 1.0 - fabs((double)(M / 2) - (double)yr * ca - (double)y);
                if (!(wz > 0.0) || !(wy > 0.0)) continue;
                const Cx<T> g = G[(p * N + x) * M + yIn];
                const double wt = wz * wy;
                re += wt * (double)g.x;
                im += wt * (double)g.y;
            }
        });
        gV[i] = Cx<T>{(T)re, (T)im};
    }
}

// Adam (Kingma & Ba, 2015), in the form with bias-corrected step and
// denominator: m <- b1 m + (1-b1) g, v <- b2 v + (1-b2) g^2,
// p <- p - (lr / c1) * m / (sqrt(v) / sqrt(c2) + eps), c_k = 1 - b_k^t.
template <typename T>
__device__ __forceinline__ void adam_apply(T& p, T g, T& m, T& v, T lr, T b1, T b2, T eps, T c1, T c2) {
    m = b1 * m + (T(1) - b1) * g;
    v = b2 * v + (T(1) - b2) * g * g;
    p -= (lr / c1) * m / (sqrt(v) / sqrt(c2) + eps);
}

// the volume as 2 * count reals (re, im interleaved), moments alike; 16-byte
// vectors (4 floats or 2 doubles) per thread and step, the tail one by one
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int N = 4;
};
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int N = 2;
};

template <typename T, bool VEC>
__global__ void k_adam_volume(T* __restrict__ V, const T* __restrict__ g, T* __restrict__ m, T* __restrict__ v,
                              uint64_t n, T lr, T b1, T b2, T eps, T c1, T c2) {
    using W = typename Vec16<T>::type;
    constexpr int K = Vec16<T>::N;
    const uint64_t nv = VEC ? n / K : 0;
    for (uint64_t i = tid_g(); i < nv; i += str_g()) {
        W pv = reinterpret_cast<W*>(V)[i], gv = reinterpret_cast<const W*>(g)[i];
        W mv = reinterpret_cast<W*>(m)[i], vv = reinterpret_cast<W*>(v)[i];
        T* pp = reinterpret_cast<T*>(&pv);
        const T* gp = reinterpret_cast<const T*>(&gv);
        T* mp = reinterpret_cast<T*>(&mv);
        T* vp = reinterpret_cast<T*>(&vv);
#pragma unroll
        for (int k = 0; k < K; ++k) adam_apply(pp[k], gp[k], mp[k], vp[k], lr, b1, b2, eps, c1, c2);
        reinterpret_cast<W*>(V)[i] = pv;
        reinterpret_cast<W*>(m)[i] = mv;
        reinterpret_cast<W*>(v)[i] = vv;
    }
    for (uint64_t i = nv * K + tid_g(); i < n; i += str_g()) adam_apply(V[i], g[i], m[i], v[i], lr, b1, b2, eps, c1, c2);
}

// angles from the per-slice sums (sums[2p + 1] = dL/d ang[p]); loss[step] =
// sum_p sums[2p] in index order (one thread: P is small)
template <typename T>
__global__ void k_adam_angles(T* __restrict__ ang, const double* __restrict__ sums, T* __restrict__ m,
                              T* __restrict__ v, uint64_t P, T lr, T b1, T b2, T eps, T c1, T c2,
                              double* __restrict__ loss) {
    for (uint64_t i = tid_g(); i < P; i += str_g())
        adam_apply(ang[i], (T)sums[2 * i + 1], m[i], v[i], lr, b1, b2, eps, c1, c2);
    if (tid_g() == 0) {
        double acc = 0.0;
        for (uint64_t p = 0; p < P; ++p) acc += sums[2 * p];
        *loss = acc;
    }
}

template <typename T>
cudaError_t refine_step_t(void* V, void* ang, const void* gV, void* mom, uint64_t vox, uint64_t P,
                          const double* sums, double lr_v, double lr_a, int step, double* loss, cudaStream_t st) {
    const T b1 = T(0.9), b2 = T(0.999), eps = T(1e-8);
    const T c1 = T(1) - pow(b1, (T)step), c2 = T(1) - pow(b2, (T)step);
    T* mv = static_cast<T*>(mom);
    const uint64_t n = 2 * vox;
    auto a16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    if (a16(V) && a16(gV) && a16(mv) && a16(mv + n))
        k_adam_volume<T, true><<<ew_grid(n / Vec16<T>::N + 1, ADJ_THREADS), ADJ_THREADS, 0, st>>>(
            static_cast<T*>(V), static_cast<const T*>(gV), mv, mv + n, n, (T)lr_v, b1, b2, eps, c1, c2);
    else
        k_adam_volume<T, false><<<ew_grid(n, ADJ_THREADS), ADJ_THREADS, 0, st>>>(
            static_cast<T*>(V), static_cast<const T*>(gV), mv, mv + n, n, (T)lr_v, b1, b2, eps, c1, c2);
    k_adam_angles<T><<<1, 128, 0, st>>>(static_cast<T*>(ang), sums, mv + 2 * n, mv + 2 * n + P, P, (T)lr_a, b1, b2,
                                        eps, c1, c2, loss);
    count_launches(2);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_refine_step(bool dbl, void* V, void* ang, const void* gV, void* moments, uint64_t vox, uint64_t P,
                               const double* sums, double lr_volume, double lr_angle, int step, double* loss,
                               cudaStream_t st) {
    return dbl ? refine_step_t<double>(V, ang, gV, moments, vox, P, sums, lr_volume, lr_angle, step, loss, st)
               : refine_step_t<float>(V, ang, gV, moments, vox, P, sums, lr_volume, lr_angle, step, loss, st);
}

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
                                   void* atab, cudaStream_t st) {
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
    if (atab && p <= (uint64_t)ANGLE_TABLE_MAX) {
        e = dbl ? launch_sort_angles<double>((const double*)ang, (int64_t)p, atab, st)
                : launch_sort_angles<float>((const float*)ang, (int64_t)p, atab, st);
        if (e != cudaSuccess) return e;
        const AngleTable t = angle_table_view(atab, (int64_t)p);
        if (dbl)
            k_slice_adjoint_w<double><<<g, ADJ_THREADS, 0, st>>>((const Cx<double>*)G, t, (Cx<double>*)gV, m, n, l);
        else
            k_slice_adjoint_w<float><<<g, ADJ_THREADS, 0, st>>>((const Cx<float>*)G, t, (Cx<float>*)gV, m, n, l);
        count_launches(3);
        return cudaGetLastError();
    }
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
