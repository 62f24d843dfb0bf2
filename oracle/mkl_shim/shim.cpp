// Project-written implementation of the oneMKL subset declared in
// oracle/mkl_shim/include (DFTI complex transforms, CBLAS ?axpby/?scal,
// mkl_malloc/mkl_free).  It exists so that the reference's own MklImpl<T>
// source (include/MKL_Impl.hpp, include/detail/MKL_Impl.inl) can be compiled
// here unchanged and used as the CPU parity oracle and CPU baseline.
// Test infrastructure only; never linked into the B200 backend.
//
// FFT: power-of-two lengths use an iterative radix-2 decimation-in-time
// transform (rows one line at a time, columns vectorised across a block of
// columns); other lengths use a direct O(n^2) DFT with an exactly reduced
// twiddle table (enough for the reference's 10x10 known-answer test and
// modest non-power-of-two sizes).  Twiddles are evaluated in long double
// (exact on the quadrant points) and rounded to T once.
#include "mkl.h"

#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <typename T>
std::complex<T> twiddle(int64_t k, int64_t n, bool inverse) {
    // exp(-i 2 pi k / n) (forward) or exp(+i 2 pi k / n) (inverse), evaluated
    // in long double with exact values on the quadrant points
    k %= n;
    if (k < 0) k += n;
    long double c, s;
    if ((4 * k) % n == 0) {
        const int q = (int)((4 * k) / n);
        const long double cq[4] = {1.0L, 0.0L, -1.0L, 0.0L};
        const long double sq[4] = {0.0L, 1.0L, 0.0L, -1.0L};
        c = cq[q]; s = sq[q];
    } else {
        const long double pi = 3.141592653589793238462643383279502884L;
        const long double a = 2.0L * pi * (long double)k / (long double)n;
        c = cosl(a); s = sinl(a);
    }
    return inverse ? std::complex<T>((T)c, (T)s) : std::complex<T>((T)c, (T)(-s));
}

bool is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }

template <typename T>
struct Line {
    int64_t n = 0;
    bool pow2 = false;
    std::vector<uint32_t> rev;              // bit reversal (pow2)
    std::vector<T> twr[2], twi[2];          // per-stage packed twiddles, [dir]
    std::vector<T> dr[2], di[2];            // direct DFT table W^k, [dir]

    void init(int64_t len) {
        n = len;
        pow2 = is_pow2(len);
        if (pow2) {
            int bits = 0;
            while ((int64_t(1) << bits) < n) ++bits;
            rev.resize(n);
            for (int64_t i = 0; i < n; ++i) {
                uint32_t r = 0;
                for (int b = 0; b < bits; ++b)
                    if (i & (int64_t(1) << b)) r |= 1u << (bits - 1 - b);
                rev[i] = r;
            }
            for (int d = 0; d < 2; ++d) {
                twr[d].clear(); twi[d].clear();
                for (int64_t len2 = 2; len2 <= n; len2 <<= 1)
                    for (int64_t j = 0; j < len2 / 2; ++j) {
                        std::complex<T> w = twiddle<T>(j, len2, d == 1);
                        twr[d].push_back(w.real());
                        twi[d].push_back(w.imag());
                    }
            }
        } else {
            for (int d = 0; d < 2; ++d) {
                dr[d].resize(n); di[d].resize(n);
                for (int64_t k = 0; k < n; ++k) {
                    std::complex<T> w = twiddle<T>(k, n, d == 1);
                    dr[d][k] = w.real(); di[d][k] = w.imag();
                }
            }
        }
    }

    // transform one contiguous line (interleaved complex)
    void run(T* a, bool inverse, T* scratch) const {
        const int d = inverse ? 1 : 0;
        if (!pow2) {
            for (int64_t f = 0; f < n; ++f) {
                T sr = 0, si = 0;
                int64_t idx = 0;
                for (int64_t t = 0; t < n; ++t) {
                    T xr = a[2 * t], xi = a[2 * t + 1];
                    T wr = dr[d][idx], wi = di[d][idx];
                    sr += xr * wr - xi * wi;
                    si += xr * wi + xi * wr;
                    idx += f;
                    if (idx >= n) idx -= n;
                }
                scratch[2 * f] = sr; scratch[2 * f + 1] = si;
            }
            std::memcpy(a, scratch, sizeof(T) * 2 * n);
            return;
        }
        for (int64_t i = 0; i < n; ++i) {
            int64_t r = rev[i];
            if (r > i) {
                std::swap(a[2 * i], a[2 * r]);
                std::swap(a[2 * i + 1], a[2 * r + 1]);
            }
        }
        const T* wr = twr[d].data();
        const T* wi = twi[d].data();
        for (int64_t len = 2; len <= n; len <<= 1) {
            const int64_t h = len / 2;
            for (int64_t i = 0; i < n; i += len) {
                T* lo = a + 2 * i;
                T* hi = a + 2 * (i + h);
                for (int64_t j = 0; j < h; ++j) {
                    T vr = hi[2 * j] * wr[j] - hi[2 * j + 1] * wi[j];
                    T vi = hi[2 * j] * wi[j] + hi[2 * j + 1] * wr[j];
                    T ur = lo[2 * j], ui = lo[2 * j + 1];
                    lo[2 * j] = ur + vr; lo[2 * j + 1] = ui + vi;
                    hi[2 * j] = ur - vr; hi[2 * j + 1] = ui - vi;
                }
            }
            wr += h; wi += h;
        }
    }

    // transform `width` interleaved lines laid out as a[row*stride + c], c<width,
    // i.e. the column direction of a row-major plane (vectorised over c)
    void run_cols(T* a, int64_t stride, int64_t width, bool inverse, T* scratch) const {
        const int d = inverse ? 1 : 0;
        if (!pow2) {
            std::vector<T> col(2 * n), out(2 * n);
            for (int64_t c = 0; c < width; ++c) {
                for (int64_t r = 0; r < n; ++r) {
                    col[2 * r] = a[r * stride + 2 * c];
                    col[2 * r + 1] = a[r * stride + 2 * c + 1];
                }
                run(col.data(), inverse, out.data());
                for (int64_t r = 0; r < n; ++r) {
                    a[r * stride + 2 * c] = col[2 * r];
                    a[r * stride + 2 * c + 1] = col[2 * r + 1];
                }
            }
            return;
        }
        (void)scratch;
        for (int64_t i = 0; i < n; ++i) {
            int64_t r = rev[i];
            if (r > i) {
                T* p = a + i * stride;
                T* q = a + r * stride;
                for (int64_t c = 0; c < 2 * width; ++c) std::swap(p[c], q[c]);
            }
        }
        const T* wr = twr[d].data();
        const T* wi = twi[d].data();
        for (int64_t len = 2; len <= n; len <<= 1) {
            const int64_t h = len / 2;
            for (int64_t i = 0; i < n; i += len) {
                for (int64_t j = 0; j < h; ++j) {
                    T* lo = a + (i + j) * stride;
                    T* hi = a + (i + j + h) * stride;
                    const T w_r = wr[j], w_i = wi[j];
                    for (int64_t c = 0; c < width; ++c) {
                        T vr = hi[2 * c] * w_r - hi[2 * c + 1] * w_i;
                        T vi = hi[2 * c] * w_i + hi[2 * c + 1] * w_r;
                        T ur = lo[2 * c], ui = lo[2 * c + 1];
                        lo[2 * c] = ur + vr; lo[2 * c + 1] = ui + vi;
                        hi[2 * c] = ur - vr; hi[2 * c + 1] = ui - vi;
                    }
                }
            }
            wr += h; wi += h;
        }
    }
};

}  // namespace

struct CpraShimDftiDesc {
    bool dbl = false;
    MKL_LONG rank = 0;
    MKL_LONG len[2] = {1, 1};
    MKL_LONG howmany = 1;
    MKL_LONG distance = 0;
    double bscale = 1.0, fscale = 1.0;
    bool committed = false;
    bool valid = true;
    Line<float> fl[2];
    Line<double> dl[2];
};

namespace {

template <typename T>
Line<T>* lines(CpraShimDftiDesc* d);
template <>
Line<float>* lines<float>(CpraShimDftiDesc* d) { return d->fl; }
template <>
Line<double>* lines<double>(CpraShimDftiDesc* d) { return d->dl; }

template <typename T>
MKL_LONG compute(CpraShimDftiDesc* d, void* inout, bool inverse) {
    T* base = static_cast<T*>(inout);
    const int64_t M = d->rank == 2 ? d->len[0] : 1;
    const int64_t N = d->rank == 2 ? d->len[1] : d->len[0];
    const int64_t plane = M * N;
    const int64_t dist = d->distance ? d->distance : plane;
    const int64_t B = d->howmany;
    Line<T>* L = lines<T>(d);
    const T scale = (T)(inverse ? d->bscale : d->fscale);
    // rows (length N, contiguous)
#pragma omp parallel
    {
        std::vector<T> scratch(2 * std::max<int64_t>(N, M) * 64);
#pragma omp for schedule(static)
        for (int64_t r = 0; r < B * M; ++r) {
            int64_t b = r / M, row = r % M;
            L[1].run(base + 2 * (b * dist + row * N), inverse, scratch.data());
        }
    }
    if (d->rank == 2 && M > 1) {
        const int64_t W = 16;
        const int64_t nblk = (N + W - 1) / W;
#pragma omp parallel
        {
            std::vector<T> scratch(2 * M);
#pragma omp for schedule(static)
            for (int64_t t = 0; t < B * nblk; ++t) {
                int64_t b = t / nblk, c0 = (t % nblk) * W;
                int64_t w = std::min<int64_t>(W, N - c0);
                L[0].run_cols(base + 2 * (b * dist + c0), 2 * N, w, inverse, scratch.data());
            }
        }
    }
    if (scale != (T)1) {
        const int64_t total = B * dist;
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b < B; ++b)
            for (int64_t i = 0; i < 2 * plane; ++i) base[2 * b * dist + i] *= scale;
        (void)total;
    }
    return DFTI_NO_ERROR;
}

}  // namespace

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* handle, DFTI_CONFIG_VALUE precision,
                              DFTI_CONFIG_VALUE domain, MKL_LONG rank, const MKL_LONG* lengths) {
    auto* d = new (std::nothrow) CpraShimDftiDesc();
    if (!d) return DFTI_INVALID_CONFIGURATION;
    *handle = d;
    d->dbl = (precision == DFTI_DOUBLE);
    d->rank = rank;
    if (domain != DFTI_COMPLEX || (rank != 1 && rank != 2)) {
        // rank 3 from a 2-length array (MKL_Impl.hpp:46-47) is refused here
        d->valid = false;
        return DFTI_UNIMPLEMENTED;
    }
    for (MKL_LONG i = 0; i < rank; ++i) d->len[i] = lengths[i];
    return DFTI_NO_ERROR;
}

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* handle, DFTI_CONFIG_VALUE precision,
                              DFTI_CONFIG_VALUE domain, MKL_LONG rank, MKL_LONG length) {
    MKL_LONG l = length;
    if (rank != 1) {
        auto* d = new CpraShimDftiDesc();
        d->valid = false;
        *handle = d;
        return DFTI_INVALID_CONFIGURATION;
    }
    return DftiCreateDescriptor(handle, precision, domain, rank, &l);
}

MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE d, DFTI_CONFIG_PARAM param, ...) {
    if (!d) return DFTI_BAD_DESCRIPTOR;
    va_list ap;
    va_start(ap, param);
    MKL_LONG st = DFTI_NO_ERROR;
    switch (param) {
        case DFTI_NUMBER_OF_TRANSFORMS: d->howmany = va_arg(ap, MKL_LONG); break;
        case DFTI_INPUT_DISTANCE:
        case DFTI_OUTPUT_DISTANCE: d->distance = va_arg(ap, MKL_LONG); break;
        case DFTI_BACKWARD_SCALE: d->bscale = va_arg(ap, double); break;  // float promotes to double
        case DFTI_FORWARD_SCALE: d->fscale = va_arg(ap, double); break;
        default: st = DFTI_UNIMPLEMENTED; break;
    }
    va_end(ap);
    return d->valid ? st : DFTI_BAD_DESCRIPTOR;
}

MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE d) {
    if (!d || !d->valid) return DFTI_BAD_DESCRIPTOR;
    const MKL_LONG M = d->rank == 2 ? d->len[0] : 1;
    const MKL_LONG N = d->rank == 2 ? d->len[1] : d->len[0];
    if (d->dbl) { d->dl[0].init(M); d->dl[1].init(N); }
    else { d->fl[0].init(M); d->fl[1].init(N); }
    d->committed = true;
    return DFTI_NO_ERROR;
}

MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE d, void* inout) {
    if (!d || !d->valid || !d->committed) return DFTI_BAD_DESCRIPTOR;
    return d->dbl ? compute<double>(d, inout, false) : compute<float>(d, inout, false);
}

MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE d, void* inout) {
    if (!d || !d->valid || !d->committed) return DFTI_BAD_DESCRIPTOR;
    return d->dbl ? compute<double>(d, inout, true) : compute<float>(d, inout, true);
}

MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE* h) {
    if (h && *h) { delete *h; *h = nullptr; }
    return DFTI_NO_ERROR;
}

MKL_LONG DftiErrorClass(MKL_LONG status, MKL_LONG error_class) { return status == error_class; }

char* DftiErrorMessage(MKL_LONG status) {
    static char ok[] = "no error";
    static char bad[] = "shim DFTI: unsupported configuration (only rank-1/rank-2 complex)";
    return status == DFTI_NO_ERROR ? ok : bad;
}

// ---- CBLAS level 1 (complex, real-or-complex scalars) ----------------------
namespace {
template <typename T>
void axpby(MKL_INT n, const void* a_, const void* x_, MKL_INT incx, const void* b_, void* y_, MKL_INT incy) {
    const T* a = static_cast<const T*>(a_);
    const T* b = static_cast<const T*>(b_);
    const T* x = static_cast<const T*>(x_);
    T* y = static_cast<T*>(y_);
    const T ar = a[0], ai = a[1], br = b[0], bi = b[1];
#pragma omp parallel for schedule(static)
    for (MKL_INT i = 0; i < n; ++i) {
        const T xr = x[2 * i * incx], xi = x[2 * i * incx + 1];
        const T yr = y[2 * i * incy], yi = y[2 * i * incy + 1];
        const T pr = ar * xr - ai * xi, pi = ar * xi + ai * xr;
        const T qr = br * yr - bi * yi, qi = br * yi + bi * yr;
        y[2 * i * incy] = pr + qr;
        y[2 * i * incy + 1] = pi + qi;
    }
}
template <typename T>
void scal(MKL_INT n, const void* a_, void* x_, MKL_INT incx) {
    const T* a = static_cast<const T*>(a_);
    T* x = static_cast<T*>(x_);
    const T ar = a[0], ai = a[1];
#pragma omp parallel for schedule(static)
    for (MKL_INT i = 0; i < n; ++i) {
        const T xr = x[2 * i * incx], xi = x[2 * i * incx + 1];
        x[2 * i * incx] = ar * xr - ai * xi;
        x[2 * i * incx + 1] = ar * xi + ai * xr;
    }
}
}  // namespace

void cblas_caxpby(MKL_INT n, const void* a, const void* x, MKL_INT incx, const void* b, void* y, MKL_INT incy) {
    axpby<float>(n, a, x, incx, b, y, incy);
}
void cblas_zaxpby(MKL_INT n, const void* a, const void* x, MKL_INT incx, const void* b, void* y, MKL_INT incy) {
    axpby<double>(n, a, x, incx, b, y, incy);
}
void cblas_cscal(MKL_INT n, const void* a, void* x, MKL_INT incx) { scal<float>(n, a, x, incx); }
void cblas_zscal(MKL_INT n, const void* a, void* x, MKL_INT incx) { scal<double>(n, a, x, incx); }

void* mkl_malloc(size_t bytes, int alignment) {
    if (alignment < 64) alignment = 64;
    size_t sz = (bytes + alignment - 1) / alignment * alignment;
    return std::aligned_alloc((size_t)alignment, sz ? sz : (size_t)alignment);
}
void mkl_free(void* p) { std::free(p); }
