// B200Impl<T>: the B200 backend behind the reference's operator interface
// CPRA::CpraImpl<T> (include/CPRA_Impl.hpp:18-63), as a drop-in next to
// CudaImpl<T> (include/CUDA_Impl.cuh) and MklImpl<T> (include/MKL_Impl.hpp).
//
// Header-only and free of CUDA headers: every operator forwards to the C ABI
// of libcpra_b200.so (include/cpra_b200.h).  Argument errors return false (the
// reference's convention, include/detail/MKL_Impl.inl:11,34,55,73,89,112);
// CUDA failures throw CPRA::b200_error, a std::runtime_error like the
// reference's CPRA::cuda_error (include/CUDA_Error_Check.hpp:29).
//
// Inside the reference tree it includes the tree's own "CPRA_Impl.hpp"; a
// backend is registered there by adding B200 to enum IMPL_TYPE
// (include/CPRA_Impl.hpp:15) and a case returning NewB200Impl<T> to
// NewCpraImpl (include/Impl_Factory.hpp:14-30).  Without the reference tree,
// define CPRA_B200_STANDALONE to use this project's restatement of the
// interface (cpra_impl_interface.hpp).
#pragma once
#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>

#ifdef CPRA_B200_STANDALONE
#include "cpra_impl_interface.hpp"
#else
#include "CPRA_Impl.hpp"
#endif
#include "../cpra_b200.h"

namespace CPRA {

struct b200_error : public std::runtime_error {
    explicit b200_error(const std::string& m) : std::runtime_error(m) {}
};

template <typename T>
class B200Impl final : public CpraImpl<T> {
    static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "B200Impl<T>: T is float or double");

  public:
    // CudaImpl(m, n, l, batch_size) (include/CUDA_Impl.cuh:16): the transform
    // shapes and batch are fixed here.
    B200Impl(uint64_t m, uint64_t n, uint64_t l, uint64_t batch_size) {
        const int dtype = std::is_same_v<T, double> ? CPRA_B200_F64 : CPRA_B200_F32;
        if (cpra_b200_create(&ctx_, dtype, m, n, l, batch_size) != CPRA_B200_OK)
            throw b200_error(std::string("cpra_b200_create: ") + cpra_b200_last_error());
    }
    B200Impl(const B200Impl&) = delete;
    B200Impl& operator=(const B200Impl&) = delete;
    ~B200Impl() override { cpra_b200_destroy(ctx_); }

    bool Initialize(T* flat_data_ptr, uint64_t num) override {
        return ok(cpra_b200_initialize(ctx_, flat_data_ptr, num), "Initialize");
    }
    bool Forward2D(std::complex<T>* flat_input) override {
        return ok(cpra_b200_forward2d(ctx_, flat_input), "Forward2D");
    }
    bool Backward2D(std::complex<T>* flat_input) override {
        return ok(cpra_b200_backward2d(ctx_, flat_input), "Backward2D");
    }
    bool FFTShift2D(std::complex<T>* flat_input, size_t M, size_t N, size_t Batch) override {
        return ok(cpra_b200_fftshift2d(ctx_, flat_input, M, N, Batch), "FFTShift2D");
    }
    bool Forward3D(std::complex<T>* flat_input) override {
        return ok(cpra_b200_forward3d(ctx_, flat_input), "Forward3D");
    }
    bool Backward3D(std::complex<T>* flat_input) override {
        return ok(cpra_b200_backward3d(ctx_, flat_input), "Backward3D");
    }
    bool FFTShift3D(std::complex<T>* flat_input, size_t M, size_t N, size_t L, size_t Batch) override {
        return ok(cpra_b200_fftshift3d(ctx_, flat_input, M, N, L, Batch), "FFTShift3D");
    }
    bool SpaceConstraint(std::complex<T>* flat_src_data, T* flat_constr_data, uint64_t num,
                         uint64_t batch_size) override {
        return ok(cpra_b200_space_constraint(ctx_, flat_src_data, flat_constr_data, num, batch_size),
                  "SpaceConstraint");
    }
    bool DataConstraint(std::complex<T>* flat_src_data, T* flat_constr_data, uint64_t num,
                        uint64_t batch_size) override {
        return ok(cpra_b200_data_constraint_real(ctx_, flat_src_data, flat_constr_data, num, batch_size),
                  "DataConstraint");
    }
    bool DataConstraint(std::complex<T>* flat_src_data, std::complex<T>* flat_constr_data, uint64_t num,
                        uint64_t batch_size) override {
        return ok(cpra_b200_data_constraint_complex(ctx_, flat_src_data, flat_constr_data, num, batch_size),
                  "DataConstraint");
    }
    bool MergeAddData(std::complex<T>* flat_src, std::complex<T>* flat_dst, T alpha, T beta, uint64_t num) override {
        return ok(cpra_b200_merge_add(ctx_, flat_src, flat_dst, alpha, beta, num), "MergeAddData");
    }
    bool Normalization(std::complex<T>* flat_src, T norm, uint64_t num) override {
        return ok(cpra_b200_normalization(ctx_, flat_src, norm, num), "Normalization");
    }
    bool Real2DTo3DInterpolation(T* flat_2d_src, T* flat_3D_dst, T* angles, uint64_t m, uint64_t n, uint64_t p,
                                 uint64_t l) override {
        return ok(cpra_b200_real2d_to_3d(ctx_, flat_2d_src, flat_3D_dst, angles, m, n, p, l),
                  "Real2DTo3DInterpolation");
    }
    bool Complex2DTo3DInterpolation(std::complex<T>* flat_2d_src, std::complex<T>* flat_3D_dst, T* angles, uint64_t m,
                                    uint64_t n, uint64_t p, uint64_t l) override {
        return ok(cpra_b200_complex2d_to_3d(ctx_, flat_2d_src, flat_3D_dst, angles, m, n, p, l),
                  "Complex2DTo3DInterpolation");
    }
    // flat_error is host memory, as include/CPRA_Impl.hpp:55 requires
    bool ConvergeError(std::complex<T>* flat_old, std::complex<T>* flat_new, T* flat_error, uint64_t m, uint64_t n,
                       uint64_t l = 1, uint64_t batch_size = 1) override {
        return ok(cpra_b200_converge_error(ctx_, flat_old, flat_new, flat_error, m, n, l, batch_size),
                  "ConvergeError");
    }
    bool Memcpy(void* dst, void* src, uint64_t bytes) override {
        return ok(cpra_b200_memcpy(ctx_, dst, src, bytes), "Memcpy");
    }
    bool Sync() override { return ok(cpra_b200_sync(ctx_), "Sync"); }

    // ---- extensions (no counterpart in CpraImpl<T>) ----
    // `iters` difference-map iterations of src/CPRA_MKL.cpp:94-110 in one launch
    bool DmIterations(std::complex<T>* x, std::complex<T>* t1, std::complex<T>* t2, T* A, T* S, uint64_t batch,
                      T beta, int iters, uint64_t a_stride = 0, uint64_t s_stride = 0) {
        return ok(cpra_b200_dm_iterations(ctx_, x, t1, t2, A, a_stride, S, s_stride, batch, beta, iters),
                  "DmIterations");
    }
    // the carousel driver of src/CPRA_MKL.cpp:35-140 on resident buffers
    bool CpraRun(std::complex<T>* x, T* A, T* S, uint64_t P, uint64_t batch, int epi, int iters, int pre_iter,
                 T beta, bool final_step, T* err_host) {
        return ok(cpra_b200_cpra_run(ctx_, x, A, S, P, batch, epi, iters, pre_iter, beta, final_step ? 1 : 0,
                                     err_host),
                  "CpraRun");
    }
    bool SetOption(int option, int64_t value) { return ok(cpra_b200_set_option(ctx_, option, value), "SetOption"); }
    void* Allocate(uint64_t bytes, bool managed = true) {
        void* p = nullptr;
        if (cpra_b200_alloc(ctx_, &p, bytes, managed ? 1 : 0) != CPRA_B200_OK)
            throw b200_error(std::string("allocate: ") + cpra_b200_last_error());
        return p;
    }
    void Deallocate(void* p) { ok(cpra_b200_free(ctx_, p), "deallocate"); }
    cpra_b200_ctx* context() const { return ctx_; }

  private:
    static bool ok(int rc, const char* what) {
        if (rc == CPRA_B200_OK) return true;
        if (rc == CPRA_B200_EARG) return false;
        throw b200_error(std::string(what) + ": " + cpra_b200_last_error());
    }
    cpra_b200_ctx* ctx_ = nullptr;
};

// factory entry, the counterpart of NewCUDAImpl / NewMKLImpl
// (include/CUDA_Impl.cuh:123-127, include/MKL_Impl.hpp:194-198)
template <typename T>
std::unique_ptr<CpraImpl<T>> NewB200Impl(uint64_t m, uint64_t n, uint64_t l, uint64_t batch_size) {
    return std::make_unique<B200Impl<T>>(m, n, l, batch_size);
}

}  // namespace CPRA
