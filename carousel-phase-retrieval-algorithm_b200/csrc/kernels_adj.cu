// Central slices of a 3D Fourier volume and the adjoints of the amplitude loss
// (project-defined; the reference has no slice operator, loss or gradient).
//
// Geometry: the merges' (CUDA_Impl_Kernel.cuh:80-90) with an in-plane rotation
// added.  A volume is [L][N][M] (y fastest); voxel (z, x, y) sits at the point
// (j, k, l) = (L/2 - z, x - N/2, M/2 - y).  Slice p has the tilt a_p (the
// merges' rotating angle) and the in-plane rotation r_p; its pixel
// (xIn, yIn), slices stored [P][N][M] (yIn fastest), has the detector
// coordinates xr = xIn - N/2, yr = M/2 - yIn, rotated in the detector plane to
//   xq = xr cos r - yr sin r,  yq = xr sin r + yr cos r,
// and sits at the point (yq sin a, xq, yq cos a), i.e. the voxel coordinates
//   zf = L/2 - yq sin a,  xf = N/2 + xq,  yf = M/2 - yq cos a.
// A slice pixel is the trilinear sample of V there,
//   s[p](xIn, yIn) = sum_{z,x,y} w(zf - z) w(xf - x) w(yf - y) V[z][x][y],
//   w(u) = max(0, 1 - |u|)   (voxels outside the volume read 0).
// With r = 0, xf = xIn is integral and the sample is the merges' bilinear
// sample on the plane x = xIn.  The plane of slice p has the normal
// (cos a, 0, -sin a) whatever r is: r turns the pixel grid inside the plane.
//
// Loss L = sum_p sum_px (|s| - A)^2 with G = 2 (|s| - A) s / |s| (0 where s = 0),
// the derivative with respect to Re s + i Im s:
//   dL/dV (Re + i Im)  = S^T G: each voxel gathers w * G from the pixels whose
//                        trilinear footprint covers it (found from the voxel's
//                        coordinates in each nearby slice's plane), so the sum
//                        is deterministic;
//   dL/da_p, dL/dr_p   = sum_px Re(conj(G) ds/da), Re(conj(G) ds/dr), from the
//                        derivatives of the weights:
//                        d(zf, xf, yf)/da = (-yq cos a, 0, yq sin a),
//                        d(zf, xf, yf)/dr = (-xq sin a, -yq, -xq cos a).
// Coordinates, weights and the per-pixel and per-voxel sums are computed in the
// element type T (float for the float path); the loss and angle-gradient sums
// over a slice's pixels are in double.  Forward and adjoint
// evaluate the same weight expression for each (pixel, voxel) pair, so the
// gather is the transpose of the sample up to the summation order.
#include "cpra_internal.h"
#include "ops_ew.cuh"
#include "angle_table.cuh"

namespace cpra_b200 {
namespace {

constexpr int ADJ_THREADS = 256;

__device__ __forceinline__ uint64_t tid_g() { return blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t str_g() { return (uint64_t)gridDim.x * blockDim.x; }

// sin and cos of a slice's tilt and in-plane rotation, in T
template <typename T>
struct Orient {
    T sa, ca, sr, cr;
};

// one entry per slice (the sines and cosines evaluated once per call, in
// double, then rounded to T); rot may be null (no in-plane rotation)
template <typename T>
__global__ void k_orient_table(const T* __restrict__ ang, const T* __restrict__ rot, Orient<T>* __restrict__ tab,
                               int64_t P) {
    for (uint64_t i = tid_g(); i < (uint64_t)P; i += str_g()) {
        const double a = (double)ang[i], r = rot ? (double)rot[i] : 0.0;
        tab[i] = Orient<T>{(T)sin(a), (T)cos(a), (T)sin(r), (T)cos(r)};
    }
}

// voxel coordinates of pixel (xr, yr) (detector coordinates) of a slice, and
// the rotated detector coordinates (xq, yq) the derivatives need
template <typename T>
__device__ __forceinline__ void pixel_point(const Orient<T>& o, T xr, T yr, T hl, T hn, T hm, T& zf, T& xf, T& yf,
                                            T& xq, T& yq) {
    xq = o.cr * xr - o.sr * yr;
    yq = o.sr * xr + o.cr * yr;
    zf = hl - yq * o.sa;
    xf = hn + xq;
    yf = hm - yq * o.ca;
}

__device__ __forceinline__ int64_t floor_i(float v) { return (int64_t)floorf(v); }
__device__ __forceinline__ int64_t floor_i(double v) { return (int64_t)floor(v); }
__device__ __forceinline__ float absT(float v) { return fabsf(v); }
__device__ __forceinline__ double absT(double v) { return fabs(v); }

// trilinear sample of V at (zf, xf, yf) and, with D, its derivatives along the
// directions (dz1, dx1, dy1) and (dz2, dx2, dy2)
template <typename T, bool D>
__device__ __forceinline__ void trilinear(const Cx<T>* __restrict__ V, int64_t M, int64_t N, int64_t L, T zf, T xf,
                                          T yf, T dz1, T dx1, T dy1, T dz2, T dx2, T dy2, T& re, T& im, T& d1r,
                                          T& d1i, T& d2r, T& d2i) {
    const int64_t z0 = floor_i(zf), x0 = floor_i(xf), y0 = floor_i(yf);
    re = im = d1r = d1i = d2r = d2i = T(0);
    for (int cz = 0; cz < 2; ++cz) {
        const int64_t z = z0 + cz;
        const T uz = zf - (T)z;
        const T wz = T(1) - absT(uz);
        if (z < 0 || z >= L || !(wz > T(0))) continue;
        const T sz = uz >= T(0) ? T(-1) : T(1);  // d wz / d zf
        for (int cx = 0; cx < 2; ++cx) {
            const int64_t x = x0 + cx;
            const T ux = xf - (T)x;
            const T wx = T(1) - absT(ux);
            if (x < 0 || x >= N || !(wx > T(0))) continue;
            const T sx = ux >= T(0) ? T(-1) : T(1);
            for (int cy = 0; cy < 2; ++cy) {
                const int64_t y = y0 + cy;
                const T uy = yf - (T)y;
                const T wy = T(1) - absT(uy);
                if (y < 0 || y >= M || !(wy > T(0))) continue;
                const T sy = uy >= T(0) ? T(-1) : T(1);
                const Cx<T> v = V[(z * N + x) * M + y];
                const T w = wz * wx * wy;
                re += w * v.x;
                im += w * v.y;
                if (D) {
                    const T g1 = sz * dz1 * wx * wy + wz * sx * dx1 * wy + wz * wx * sy * dy1;
                    const T g2 = sz * dz2 * wx * wy + wz * sx * dx2 * wy + wz * wx * sy * dy2;
                    d1r += g1 * v.x;
                    d1i += g1 * v.y;
                    d2r += g2 * v.x;
                    d2i += g2 * v.y;
                }
            }
        }
    }
}

template <typename T>
__global__ void k_slice(const Cx<T>* __restrict__ V, const Orient<T>* __restrict__ tab, Cx<T>* __restrict__ out,
                        int64_t M, int64_t N, int64_t P, int64_t L) {
    const uint64_t total = (uint64_t)P * N * M;
    const T hl = (T)(L / 2), hn = (T)(N / 2), hm = (T)(M / 2);
    for (uint64_t i = tid_g(); i < total; i += str_g()) {
        const int64_t yIn = (int64_t)(i % M), xIn = (int64_t)((i / M) % N), p = (int64_t)(i / ((uint64_t)M * N));
        const Orient<T> o = tab[p];
        T zf, xf, yf, xq, yq;
        pixel_point(o, (T)(xIn - N / 2), (T)(M / 2 - yIn), hl, hn, hm, zf, xf, yf, xq, yq);
        T re, im, a, b, c, d;
        const T z0 = T(0);
        trilinear<T, false>(V, M, N, L, zf, xf, yf, z0, z0, z0, z0, z0, z0, re, im, a, b, c, d);
        out[i] = Cx<T>{re, im};
    }
}

// G and the per-slice sums of the loss and of Re(conj(G) ds/da),
// Re(conj(G) ds/dr); grid (CONVERGE_BLOCKS, P), one partial triple per block
template <typename T>
__global__ void k_slice_residual(const Cx<T>* __restrict__ V, const Orient<T>* __restrict__ tab,
                                 const T* __restrict__ A, Cx<T>* __restrict__ G, int64_t M, int64_t N, int64_t L,
                                 double* __restrict__ partials) {
    __shared__ double sl[ADJ_THREADS], sg[ADJ_THREADS], sh[ADJ_THREADS];
    const int64_t p = blockIdx.y;
    const Orient<T> o = tab[p];
    const uint64_t plane = (uint64_t)N * M;
    const T hl = (T)(L / 2), hn = (T)(N / 2), hm = (T)(M / 2);
    double accL = 0.0, accA = 0.0, accR = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)ADJ_THREADS + threadIdx.x; i < plane; i += (uint64_t)gridDim.x * ADJ_THREADS) {
        const int64_t yIn = (int64_t)(i % M), xIn = (int64_t)(i / M);
        T zf, xf, yf, xq, yq;
        pixel_point(o, (T)(xIn - N / 2), (T)(M / 2 - yIn), hl, hn, hm, zf, xf, yf, xq, yq);
        T ret, imt, dart, dait, drrt, drit;
        trilinear<T, true>(V, M, N, L, zf, xf, yf, -yq * o.ca, T(0), yq * o.sa, -xq * o.sa, -yq, -xq * o.ca, ret, imt,
                           dart, dait, drrt, drit);
        // the per-pixel terms of the loss and angle sums in double (they are summed over the plane)
        const double re = ret, im = imt, dar = dart, dai = dait, drr = drrt, dri = drit;
        const double mag = sqrt(re * re + im * im);
        const double d = mag - (double)A[p * plane + i];
        accL += d * d;
        double gr = 0.0, gi = 0.0;
        if (mag > 0.0) {
            gr = 2.0 * d * re / mag;
            gi = 2.0 * d * im / mag;
        }
        G[p * plane + i] = Cx<T>{(T)gr, (T)gi};
        accA += gr * dar + gi * dai;
        accR += gr * drr + gi * dri;
    }
    sl[threadIdx.x] = accL;
    sg[threadIdx.x] = accA;
    sh[threadIdx.x] = accR;
    __syncthreads();
    for (int h = ADJ_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sl[threadIdx.x] += sl[threadIdx.x + h];
            sg[threadIdx.x] += sg[threadIdx.x + h];
            sh[threadIdx.x] += sh[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* q = partials + (p * gridDim.x + blockIdx.x) * 3;
        q[0] = sl[0];
        q[1] = sg[0];
        q[2] = sh[0];
    }
}

// sums[3p + c] = the CONVERGE_BLOCKS partials of slice p, in block order
__global__ void k_sum3_final(const double* __restrict__ partials, double* __restrict__ sums, int64_t P) {
    for (uint64_t i = tid_g(); i < (uint64_t)P * 3; i += str_g()) {
        const uint64_t p = i / 3, c = i % 3;
        double acc = 0.0;
        for (int b = 0; b < CONVERGE_BLOCKS; ++b) acc += partials[(p * CONVERGE_BLOCKS + b) * 3 + c];
        sums[i] = acc;
    }
}

// the adjoint's contribution of slice p to the voxel at point (j, k, l), voxel
// indices (z, x, y): the pixels whose trilinear footprint covers the voxel.
// In the slice's plane the voxel has the coordinates u = k (along the tilt
// axis) and v = j sin a + l cos a, and the distance d = j cos a - l sin a.  A
// pixel covers it only if |d| < sqrt 2 and its rotated coordinates satisfy
// |xq - u| < 1, |yq - v| < sqrt 2; turned back by -r that rectangle bounds the
// candidate (xr, yr), whose weight is then computed as in the forward sample.
constexpr double ADJ_SQRT2 = 1.4142135623730951;
// the pixels part: (u, v) the voxel's in-plane coordinates before the
// rotation (u = k along the tilt axis, v from the voxel's (j, l) only)
template <typename T>
__device__ __forceinline__ void gather_pixels(const Cx<T>* __restrict__ Gp, const Orient<T>& o, int64_t M, int64_t N,
                                              T hl, T hn, T hm, T u, T v, int64_t z, int64_t x, int64_t y, T& re,
                                              T& im) {
    const T xc = o.cr * u + o.sr * v, yc = o.cr * v - o.sr * u;
    const T ar = absT(o.cr), as = absT(o.sr);
    const T hx = ar + as * T(ADJ_SQRT2) + T(1e-3), hy = as + ar * T(ADJ_SQRT2) + T(1e-3);
    // 32-bit window and pixel indices (a slice is at most 2^31 pixels)
    const int m = (int)M, n = (int)N;
    const int xr0 = (int)floor_i(xc - hx) + 1, xr1 = (int)floor_i(xc + hx);
    const int yr0 = (int)floor_i(yc - hy) + 1, yr1 = (int)floor_i(yc + hy);
    for (int xr = xr0; xr <= xr1; ++xr) {
        const int xIn = xr + n / 2;
        if (xIn < 0 || xIn >= n) continue;
        for (int yr = yr0; yr <= yr1; ++yr) {
            const int yIn = m / 2 - yr;
            if (yIn < 0 || yIn >= m) continue;
            T zf, xf, yf, xq, yq;
            pixel_point(o, (T)xr, (T)yr, hl, hn, hm, zf, xf, yf, xq, yq);
            const T wz = T(1) - absT(zf - (T)z), wx = T(1) - absT(xf - (T)x), wy = T(1) - absT(yf - (T)y);
            if (!(wz > T(0)) || !(wx > T(0)) || !(wy > T(0))) continue;
            const Cx<T> g = Gp[xIn * m + yIn];
            const T w = wz * wx * wy;
            re += w * g.x;
            im += w * g.y;
        }
    }
}
// the plane part first: the slice's distance d from the voxel's point (j, l)
// decides whether the slice can reach it at all
template <typename T>
__device__ __forceinline__ bool gather_plane(const Orient<T>& o, T j, T l, T& v) {
    const T d = j * o.ca - l * o.sa;
    if (!(absT(d) < T(ADJ_SQRT2 + 1e-3))) return false;
    v = j * o.sa + l * o.ca;
    return true;
}
template <typename T>
__device__ __forceinline__ void gather_slice(const Cx<T>* __restrict__ Gp, const Orient<T>& o, int64_t M, int64_t N,
                                             T hl, T hn, T hm, T j, T k, T l, int64_t z, int64_t x, int64_t y, T& re,
                                             T& im) {
    T v;
    if (gather_plane(o, j, l, v)) gather_pixels(Gp, o, M, N, hl, hn, hm, k, v, z, x, y, re, im);
}

// gradient with respect to V, every slice visited (more slices than the
// direction table holds)
template <typename T>
__global__ void __launch_bounds__(ADJ_THREADS) k_slice_adjoint(const Cx<T>* __restrict__ G,
                                                               const Orient<T>* __restrict__ tab,
                                                               Cx<T>* __restrict__ gV, int64_t M, int64_t N,
                                                               int64_t P, int64_t L) {
    const uint64_t total = (uint64_t)L * N * M;
    const T hl = (T)(L / 2), hn = (T)(N / 2), hm = (T)(M / 2);
    for (uint64_t i = tid_g(); i < total; i += str_g()) {
        const int64_t y = (int64_t)(i % M), x = (int64_t)((i / M) % N), z = (int64_t)(i / ((uint64_t)M * N));
        const T j = (T)(L / 2 - z), k = (T)(x - N / 2), l = (T)(M / 2 - y);
        T re = T(0), im = T(0);
        for (int64_t p = 0; p < P; ++p)
            gather_slice(G + p * N * M, tab[p], M, N, hl, hn, hm, j, k, l, z, x, y, re, im);
        gV[i] = Cx<T>{re, im};
    }
}

// the same gather visiting only the slices whose plane passes near the voxel
// (angle_table.cuh: ordered by tilt, which alone fixes the plane), in
// direction order; voxels handed out dynamically (their cost varies with
// the distance from the tilt axis)
// XC voxels along the tilt axis per work item at one (z, y): the slices near
// them and each slice's plane part depend only on (z, y), so they are found
// once for the item; each voxel sums its slices' pixels in the same order as
// alone.  Consecutive items take consecutive y (coalesced reads and stores).
// Two voxels per item pay where the slices are dense (a voxel then has many
// candidates): measured 21.5 -> 19.7 ms at 512^3 x 720 slices, but 1.51 ->
// 1.68 ms at 256^3 x 180, so from ADJ_XC2_SLICES slices on (between the two).
constexpr int ADJ_XC2_SLICES = 360;
template <typename T, int XC>
__global__ void __launch_bounds__(ADJ_THREADS) k_slice_adjoint_w(const Cx<T>* __restrict__ G, const AngleTable at,
                                                                 const Orient<T>* __restrict__ tab,
                                                                 Cx<T>* __restrict__ gV, int64_t M, int64_t N,
                                                                 int64_t L) {
    const int64_t chunks = N / XC;
    const uint64_t total = (uint64_t)L * chunks * M;
    const T hl = (T)(L / 2), hn = (T)(N / 2), hm = (T)(M / 2);
    const bool narrow = total <= 0xffffffffull;  // 32-bit index arithmetic
    for_voxels_dynamic(at.next, total, [&](uint64_t i) {
        int64_t y, c, z;
        if (narrow) {
            const uint32_t i32 = (uint32_t)i, m32 = (uint32_t)M, c32 = (uint32_t)chunks, q = i32 / m32;
            y = (int64_t)(i32 - q * m32);
            c = (int64_t)(q % c32);
            z = (int64_t)(q / c32);
        } else {
            y = (int64_t)(i % M);
            c = (int64_t)((i / M) % chunks);
            z = (int64_t)(i / ((uint64_t)M * chunks));
        }
        const int64_t x0 = c * XC;
        const T j = (T)(L / 2 - z), l = (T)(M / 2 - y);
        T re[XC], im[XC];
#pragma unroll
        for (int t = 0; t < XC; ++t) re[t] = im[t] = T(0);
        for_slices_near(at, (double)(L / 2 - z), (double)(M / 2 - y), [&](int64_t p, double, double) {
            const Orient<T> o = tab[p];
            T v;
            if (!gather_plane(o, j, l, v)) return;
            const Cx<T>* __restrict__ Gp = G + p * N * M;
#pragma unroll
            for (int t = 0; t < XC; ++t)
                gather_pixels(Gp, o, M, N, hl, hn, hm, (T)(x0 + t - N / 2), v, z, x0 + t, y, re[t], im[t]);
        });
#pragma unroll
        for (int t = 0; t < XC; ++t) gV[((uint64_t)z * N + x0 + t) * M + y] = Cx<T>{re[t], im[t]};
    });
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
    uint64_t nv = 0;
    if constexpr (VEC) {
        nv = n / K;
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
    }
    for (uint64_t i = nv * K + tid_g(); i < n; i += str_g()) adam_apply(V[i], g[i], m[i], v[i], lr, b1, b2, eps, c1, c2);
}

// tilts and rotations from the per-slice sums (sums[3p + 1] = dL/da_p,
// sums[3p + 2] = dL/dr_p); rot may be null (not refined).  loss = sum_p
// sums[3p] in index order (one thread: P is small)
template <typename T>
__global__ void k_adam_angles(T* __restrict__ ang, T* __restrict__ rot, const double* __restrict__ sums,
                              T* __restrict__ mom, uint64_t P, T lr_a, T lr_r, T b1, T b2, T eps, T c1, T c2,
                              double* __restrict__ loss) {
    for (uint64_t i = tid_g(); i < P; i += str_g()) {
        adam_apply(ang[i], (T)sums[3 * i + 1], mom[i], mom[P + i], lr_a, b1, b2, eps, c1, c2);
        if (rot) adam_apply(rot[i], (T)sums[3 * i + 2], mom[2 * P + i], mom[3 * P + i], lr_r, b1, b2, eps, c1, c2);
    }
    if (tid_g() == 0) {
        double acc = 0.0;
        for (uint64_t p = 0; p < P; ++p) acc += sums[3 * p];
        *loss = acc;
    }
}

// volume parameters: `nv` reals (2 * voxels for a complex Fourier volume, the
// voxels of a real volume); moments: 2 nv for them, then 4 P for the angles
template <typename T>
cudaError_t refine_step_t(void* V, uint64_t nv, void* ang, void* rot, const void* gV, void* mom, uint64_t P,
                          const double* sums, double lr_v, double lr_a, double lr_r, int step, double* loss,
                          cudaStream_t st) {
    const T b1 = T(0.9), b2 = T(0.999), eps = T(1e-8);
    const T c1 = T(1) - pow(b1, (T)step), c2 = T(1) - pow(b2, (T)step);
    T* mv = static_cast<T*>(mom);
    const uint64_t n = nv;
    auto a16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    if (a16(V) && a16(gV) && a16(mv) && a16(mv + n))
        k_adam_volume<T, true><<<ew_grid(n / Vec16<T>::N + 1, ADJ_THREADS), ADJ_THREADS, 0, st>>>(
            static_cast<T*>(V), static_cast<const T*>(gV), mv, mv + n, n, (T)lr_v, b1, b2, eps, c1, c2);
    else
        k_adam_volume<T, false><<<ew_grid(n, ADJ_THREADS), ADJ_THREADS, 0, st>>>(
            static_cast<T*>(V), static_cast<const T*>(gV), mv, mv + n, n, (T)lr_v, b1, b2, eps, c1, c2);
    k_adam_angles<T><<<1, 128, 0, st>>>(static_cast<T*>(ang), static_cast<T*>(rot), sums, mv + 2 * n, P, (T)lr_a,
                                        (T)lr_r, b1, b2, eps, c1, c2, loss);
    count_launches(2);
    return cudaGetLastError();
}

// a real volume as complex values (imaginary parts 0), and back: the real
// parts times `scale`
template <typename T>
__global__ void k_real_to_complex(const T* __restrict__ r, Cx<T>* __restrict__ c, uint64_t n) {
    for (uint64_t i = tid_g(); i < n; i += str_g()) c[i] = Cx<T>{r[i], T(0)};
}
template <typename T>
__global__ void k_complex_real_part(const Cx<T>* __restrict__ c, T* __restrict__ r, T scale, uint64_t n) {
    for (uint64_t i = tid_g(); i < n; i += str_g()) r[i] = c[i].x * scale;
}

template <typename T>
cudaError_t slice_loss_grad_t(const void* V, const void* ang, const void* tab, const void* A, void* G, void* gV,
                              uint64_t m, uint64_t n, uint64_t p, uint64_t l, double* partials, double* sums,
                              void* atab, cudaStream_t st) {
    dim3 grid(CONVERGE_BLOCKS, (unsigned)p);
    k_slice_residual<T><<<grid, ADJ_THREADS, 0, st>>>((const Cx<T>*)V, (const Orient<T>*)tab, (const T*)A,
                                                       (Cx<T>*)G, m, n, l, partials);
    k_sum3_final<<<ew_grid(3 * p, ADJ_THREADS), ADJ_THREADS, 0, st>>>(partials, sums, (int64_t)p);
    count_launches(2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const uint64_t vox = l * n * m;
    const unsigned g = ew_grid(vox, ADJ_THREADS);
    if (atab && p <= (uint64_t)ANGLE_TABLE_MAX) {
        e = launch_sort_angles<T>((const T*)ang, (int64_t)p, atab, st);
        if (e != cudaSuccess) return e;
        const AngleTable t = angle_table_view(atab, (int64_t)p);
        e = cudaMemsetAsync(t.next, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
        if (p >= (uint64_t)ADJ_XC2_SLICES && n % 2 == 0)
            k_slice_adjoint_w<T, 2><<<resident_grid(k_slice_adjoint_w<T, 2>, ADJ_THREADS), ADJ_THREADS, 0, st>>>(
                (const Cx<T>*)G, t, (const Orient<T>*)tab, (Cx<T>*)gV, m, n, l);
        else
            k_slice_adjoint_w<T, 1><<<resident_grid(k_slice_adjoint_w<T, 1>, ADJ_THREADS), ADJ_THREADS, 0, st>>>(
                (const Cx<T>*)G, t, (const Orient<T>*)tab, (Cx<T>*)gV, m, n, l);
        count_launches(2);
        return cudaGetLastError();
    }
    k_slice_adjoint<T><<<g, ADJ_THREADS, 0, st>>>((const Cx<T>*)G, (const Orient<T>*)tab, (Cx<T>*)gV, m, n, p, l);
    count_launches();
    return cudaGetLastError();
}

}  // namespace

uint64_t orient_table_bytes(bool dbl, uint64_t p) { return p * (dbl ? sizeof(Orient<double>) : sizeof(Orient<float>)); }

cudaError_t launch_orient_table(bool dbl, const void* ang, const void* rot, void* tab, uint64_t p, cudaStream_t st) {
    if (p == 0) return cudaSuccess;
    const unsigned g = ew_grid(p, ADJ_THREADS);
    if (dbl)
        k_orient_table<double><<<g, ADJ_THREADS, 0, st>>>((const double*)ang, (const double*)rot,
                                                          (Orient<double>*)tab, (int64_t)p);
    else
        k_orient_table<float><<<g, ADJ_THREADS, 0, st>>>((const float*)ang, (const float*)rot, (Orient<float>*)tab,
                                                         (int64_t)p);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_refine_step(bool dbl, void* V, uint64_t nv, void* ang, void* rot, const void* gV, void* moments,
                               uint64_t P, const double* sums, double lr_volume, double lr_angle, double lr_rot,
                               int step, double* loss, cudaStream_t st) {
    return dbl ? refine_step_t<double>(V, nv, ang, rot, gV, moments, P, sums, lr_volume, lr_angle, lr_rot, step, loss,
                                       st)
               : refine_step_t<float>(V, nv, ang, rot, gV, moments, P, sums, lr_volume, lr_angle, lr_rot, step, loss,
                                      st);
}

cudaError_t launch_slice(bool dbl, const void* V, const void* tab, void* out, uint64_t m, uint64_t n, uint64_t p,
                         uint64_t l, cudaStream_t st) {
    const uint64_t total = p * n * m;
    if (total == 0) return cudaSuccess;
    const unsigned g = ew_grid(total, ADJ_THREADS);
    if (dbl)
        k_slice<double><<<g, ADJ_THREADS, 0, st>>>((const Cx<double>*)V, (const Orient<double>*)tab,
                                                   (Cx<double>*)out, m, n, p, l);
    else
        k_slice<float><<<g, ADJ_THREADS, 0, st>>>((const Cx<float>*)V, (const Orient<float>*)tab, (Cx<float>*)out, m,
                                                  n, p, l);
    count_launches();
    return cudaGetLastError();
}

cudaError_t launch_slice_loss_grad(bool dbl, const void* V, const void* ang, const void* tab, const void* A, void* G,
                                   void* gV, uint64_t m, uint64_t n, uint64_t p, uint64_t l, double* partials,
                                   double* sums, void* atab, cudaStream_t st) {
    if (p == 0) return cudaSuccess;
    if (p > 65535) return cudaErrorInvalidValue;
    return dbl ? slice_loss_grad_t<double>(V, ang, tab, A, G, gV, m, n, p, l, partials, sums, atab, st)
               : slice_loss_grad_t<float>(V, ang, tab, A, G, gV, m, n, p, l, partials, sums, atab, st);
}

cudaError_t launch_real_complex(bool dbl, bool to_complex, void* real, void* cplx, double scale, uint64_t n,
                                cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const unsigned g = ew_grid(n, ADJ_THREADS);
    if (to_complex) {
        if (dbl)
            k_real_to_complex<double><<<g, ADJ_THREADS, 0, st>>>((const double*)real, (Cx<double>*)cplx, n);
        else
            k_real_to_complex<float><<<g, ADJ_THREADS, 0, st>>>((const float*)real, (Cx<float>*)cplx, n);
    } else {
        if (dbl)
            k_complex_real_part<double><<<g, ADJ_THREADS, 0, st>>>((const Cx<double>*)cplx, (double*)real, scale, n);
        else
            k_complex_real_part<float><<<g, ADJ_THREADS, 0, st>>>((const Cx<float>*)cplx, (float*)real,
                                                                  (float)scale, n);
    }
    count_launches();
    return cudaGetLastError();
}

}  // namespace cpra_b200
