// extern "C" access to the reference's own operator backend MklImpl<T>
// (include/MKL_Impl.hpp, include/detail/MKL_Impl.inl), compiled unchanged from
// the reference's include directory against the project's DFTI/CBLAS shim
// (oracle/mkl_shim).  Test infrastructure only: the parity tests, the golden
// fixture generator and the CPU-baseline leg of bench.py call it through
// ctypes; the B200 backend never links it.
//
// Besides one wrapper per operator it restates the reference's driver loops
// (src/CPRA_MKL.cpp:35-140) as functions that take seeded initial guesses
// instead of the reference's unseeded Initialize() fill, so that identical
// inputs can be given to the numpy oracle, these compiled reference operators
// and the B200 backend.
// The reference reaches MKL_Impl.hpp through CPRA.hpp, which includes these
// first (include/CPRA.hpp:2-5); MKL_Impl.hpp relies on them.
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>

#include "MKL_Impl.hpp"

#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <typename T>
using Impl = CPRA::MklImpl<T>;

template <typename T>
Impl<T>* H(void* h) { return static_cast<Impl<T>*>(h); }

#define CPRA_REF_DISPATCH(dbl, EXPR_F, EXPR_D) ((dbl) ? (EXPR_D) : (EXPR_F))

// src/CPRA_MKL.cpp:94-110: one difference-map iteration in the driver's order,
// with its coefficient expressions (double arithmetic on a T beta, passed as T)
template <typename T>
void dm_iteration(Impl<T>* impl, std::complex<T>* x, std::complex<T>* t1, std::complex<T>* t2,
                  T* A, T* S, uint64_t num, uint64_t batch, T Beta) {
    impl->Forward2D(t1);
    impl->DataConstraint(t1, A, num, batch);
    impl->Backward2D(t1);
    impl->MergeAddData(x, t1, -1.0 / Beta, 1.0 + 1.0 / Beta, num);
    impl->SpaceConstraint(t1, S, num, batch);
    impl->SpaceConstraint(t2, S, num, batch);
    impl->MergeAddData(x, t2, 1.0 / Beta, 1.0 - 1.0 / Beta, num);
    impl->Forward2D(t2);
    impl->DataConstraint(t2, A, num, batch);
    impl->Backward2D(t2);
    impl->MergeAddData(t1, x, Beta, 1.0, num);
    impl->MergeAddData(t2, x, -1.0 * Beta, 1.0, num);
}

// src/CPRA_MKL.cpp:35-140 with x supplied by the caller ([P][B][M][N]).
template <typename T>
void cpra_sample(uint64_t M, uint64_t N, uint64_t L, uint64_t P, uint64_t B, T* A, T* S,
                 std::complex<T>* x, int epi, int iter, int pre_iter, T Beta, T* err) {
    Impl<T> impl(M, N, L, B);
    const uint64_t MNB = M * N * B;
    std::complex<T>* t1 = new std::complex<T>[MNB];
    std::complex<T>* t2 = new std::complex<T>[MNB];
    std::complex<T>* old = new std::complex<T>[MNB];
    const size_t bytes = sizeof(std::complex<T>) * MNB;
    // MklImpl::Memcpy has no return statement (MKL_Impl.hpp:159-162), so the
    // copies are done with std::memcpy, which is all it would do
    std::memcpy(t1, x, bytes);
    std::memcpy(t2, x, bytes);
    for (int i = 0; i < pre_iter; ++i) dm_iteration<T>(&impl, x, t1, t2, A, S, MNB, B, Beta);
    for (int e = 0; e < epi; ++e) {
        for (uint64_t p = 0; p < P; ++p) {
            std::complex<T>* xp = x + MNB * p;
            if (p == P - 1) {
                impl.MergeAddData(x + MNB * (p - 1), xp, 0.5, 0.5, MNB);
            } else if (p == 0) {
                impl.MergeAddData(x + MNB * (p + 1), xp, 0.5, 0.5, MNB);
            } else {
                impl.MergeAddData(x + MNB * (p - 1), xp, 0.5, 0, MNB);
                impl.MergeAddData(x + MNB * (p + 1), xp, 0.5, 1, MNB);
            }
            std::memcpy(t1, xp, bytes);
            std::memcpy(t2, xp, bytes);
            for (int i = 0; i < iter; ++i) {
                const bool last = (i == iter - 1 && e == epi - 1);
                if (last) std::memcpy(old, xp, bytes);
                dm_iteration<T>(&impl, xp, t1, t2, A + M * N * p, S + M * N * p, MNB, B, Beta);
                if (last) {
                    std::memcpy(t1, xp, bytes);
                    impl.Forward2D(old);
                    impl.Forward2D(t1);
                    // stub in the MKL backend (MKL_Impl.hpp:154-157): err untouched
                    impl.ConvergeError(old, t1, err + B * p, M, N, 1, B);
                }
            }
        }
    }
    for (uint64_t p = 0; p < P; ++p) {
        std::complex<T>* xp = x + MNB * p;
        std::memcpy(t1, xp, bytes);
        impl.Forward2D(t1);
        impl.DataConstraint(t1, A + M * N * p, MNB, B);
        impl.Backward2D(t1);
        impl.MergeAddData(xp, t1, -1.0 / Beta, 1.0 + 1.0 / Beta, MNB);
        impl.SpaceConstraint(t1, S + M * N * p, MNB, B);
        std::memcpy(xp, t1, bytes);
    }
    delete[] t1;
    delete[] t2;
    delete[] old;
}

}  // namespace

extern "C" {

void* cpra_ref_create(int dbl, uint64_t m, uint64_t n, uint64_t l, uint64_t batch) {
    if (dbl) return new Impl<double>(m, n, l, batch);
    return new Impl<float>(m, n, l, batch);
}

void cpra_ref_destroy(int dbl, void* h) {
    if (dbl) delete H<double>(h);
    else delete H<float>(h);
}

int cpra_ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int cpra_ref_forward2d(int dbl, void* h, void* x) {
    return CPRA_REF_DISPATCH(dbl, H<float>(h)->Forward2D((std::complex<float>*)x),
                             H<double>(h)->Forward2D((std::complex<double>*)x));
}
int cpra_ref_backward2d(int dbl, void* h, void* x) {
    return CPRA_REF_DISPATCH(dbl, H<float>(h)->Backward2D((std::complex<float>*)x),
                             H<double>(h)->Backward2D((std::complex<double>*)x));
}
int cpra_ref_fftshift2d(int dbl, void* h, void* x, uint64_t M, uint64_t N, uint64_t B) {
    return CPRA_REF_DISPATCH(dbl, H<float>(h)->FFTShift2D((std::complex<float>*)x, M, N, B),
                             H<double>(h)->FFTShift2D((std::complex<double>*)x, M, N, B));
}
int cpra_ref_fftshift3d(int dbl, void* h, void* x, uint64_t M, uint64_t N, uint64_t L, uint64_t B) {
    return CPRA_REF_DISPATCH(dbl, H<float>(h)->FFTShift3D((std::complex<float>*)x, M, N, L, B),
                             H<double>(h)->FFTShift3D((std::complex<double>*)x, M, N, L, B));
}
int cpra_ref_space_constraint(int dbl, void* h, void* x, void* s, uint64_t num, uint64_t batch) {
    return CPRA_REF_DISPATCH(dbl, H<float>(h)->SpaceConstraint((std::complex<float>*)x, (float*)s, num, batch),
                             H<double>(h)->SpaceConstraint((std::complex<double>*)x, (double*)s, num, batch));
}
int cpra_ref_data_constraint_real(int dbl, void* h, void* x, void* a, uint64_t num, uint64_t batch) {
    return CPRA_REF_DISPATCH(dbl, H<float>(h)->DataConstraint((std::complex<float>*)x, (float*)a, num, batch),
                             H<double>(h)->DataConstraint((std::complex<double>*)x, (double*)a, num, batch));
}
int cpra_ref_data_constraint_complex(int dbl, void* h, void* x, void* c, uint64_t num, uint64_t batch) {
    return CPRA_REF_DISPATCH(
        dbl, H<float>(h)->DataConstraint((std::complex<float>*)x, (std::complex<float>*)c, num, batch),
        H<double>(h)->DataConstraint((std::complex<double>*)x, (std::complex<double>*)c, num, batch));
}
int cpra_ref_merge_add(int dbl, void* h, void* src, void* dst, double alpha, double beta, uint64_t num) {
    return CPRA_REF_DISPATCH(
        dbl, H<float>(h)->MergeAddData((std::complex<float>*)src, (std::complex<float>*)dst, (float)alpha, (float)beta, num),
        H<double>(h)->MergeAddData((std::complex<double>*)src, (std::complex<double>*)dst, alpha, beta, num));
}
int cpra_ref_normalization(int dbl, void* h, void* x, double norm, uint64_t num) {
    return CPRA_REF_DISPATCH(dbl, H<float>(h)->Normalization((std::complex<float>*)x, (float)norm, num),
                             H<double>(h)->Normalization((std::complex<double>*)x, norm, num));
}
int cpra_ref_initialize(int dbl, void* h, void* x, uint64_t num) {
    return CPRA_REF_DISPATCH(dbl, H<float>(h)->Initialize((float*)x, num),
                             H<double>(h)->Initialize((double*)x, num));
}

// `iters` difference-map iterations on one batch (src/CPRA_MKL.cpp:94-110)
int cpra_ref_dm_iterations(int dbl, void* h, void* x, void* t1, void* t2, void* A, void* S,
                           uint64_t num, uint64_t batch, double beta, int iters) {
    for (int i = 0; i < iters; ++i) {
        if (dbl)
            dm_iteration<double>(H<double>(h), (std::complex<double>*)x, (std::complex<double>*)t1,
                                 (std::complex<double>*)t2, (double*)A, (double*)S, num, batch, beta);
        else
            dm_iteration<float>(H<float>(h), (std::complex<float>*)x, (std::complex<float>*)t1,
                                (std::complex<float>*)t2, (float*)A, (float*)S, num, batch, (float)beta);
    }
    return 1;
}

int cpra_ref_cpra_sample(int dbl, uint64_t M, uint64_t N, uint64_t L, uint64_t P, uint64_t B, void* A,
                         void* S, void* x, int epi, int iter, int pre_iter, double beta, void* err) {
    if (P < 2) return 0;  // the carousel mix reads angle p-1 / p+1
    if (dbl)
        cpra_sample<double>(M, N, L, P, B, (double*)A, (double*)S, (std::complex<double>*)x, epi, iter,
                            pre_iter, beta, (double*)err);
    else
        cpra_sample<float>(M, N, L, P, B, (float*)A, (float*)S, (std::complex<float>*)x, epi, iter, pre_iter,
                           (float)beta, (float*)err);
    return 1;
}

}  // extern "C"
