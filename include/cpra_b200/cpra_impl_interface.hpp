// The operator interface CPRA::CpraImpl<T>, restated for builds of the B200
// backend outside the reference tree (define CPRA_B200_STANDALONE).  The
// virtuals, their order, parameter types and defaults are the reference's
// (include/CPRA_Impl.hpp:18-63) so that code written against either compiles
// unchanged; inside the reference tree its own CPRA_Impl.hpp is used instead.
#pragma once
#include <complex>
#include <cstddef>
#include <cstdint>

namespace CPRA {

enum IMPL_TYPE { CUDA, MKL, B200 };

template <typename T>
class CpraImpl {
  public:
    CpraImpl() {}
    virtual bool Initialize(T* flat_data_ptr, uint64_t num) = 0;
    virtual bool Forward2D(std::complex<T>* flat_input) = 0;
    virtual bool Backward2D(std::complex<T>* flat_input) = 0;
    virtual bool FFTShift2D(std::complex<T>* flat_input, size_t M, size_t N, size_t Batch) = 0;
    virtual bool Forward3D(std::complex<T>* flat_input) = 0;
    virtual bool Backward3D(std::complex<T>* flat_input) = 0;
    virtual bool FFTShift3D(std::complex<T>* flat_input, size_t M, size_t N, size_t L, size_t Batch) = 0;
    virtual bool SpaceConstraint(std::complex<T>* flat_src_data, T* flat_constr_data, uint64_t num,
                                 uint64_t batch_size) = 0;
    virtual bool DataConstraint(std::complex<T>* flat_src_data, T* flat_constr_data, uint64_t num,
                                uint64_t batch_size) = 0;
    virtual bool DataConstraint(std::complex<T>* flat_src_data, std::complex<T>* flat_constr_data, uint64_t num,
                                uint64_t batch_size) = 0;
    virtual bool MergeAddData(std::complex<T>* flat_src, std::complex<T>* flat_dst, T alpha, T beta,
                              uint64_t num) = 0;
    virtual bool Normalization(std::complex<T>* flat_src, T norm, uint64_t num) = 0;
    virtual bool Real2DTo3DInterpolation(T* flat_2d_src, T* flat_3D_dst, T* angles, uint64_t m, uint64_t n,
                                         uint64_t p, uint64_t l) = 0;
    virtual bool Complex2DTo3DInterpolation(std::complex<T>* flat_2d_src, std::complex<T>* flat_3D_dst, T* angles,
                                            uint64_t m, uint64_t n, uint64_t p, uint64_t l) = 0;
    virtual bool ConvergeError(std::complex<T>* flat_old, std::complex<T>* flat_new, T* flat_error, uint64_t m,
                               uint64_t n, uint64_t l = 1, uint64_t batch_size = 1) = 0;
    virtual bool Memcpy(void* dst, void* src, uint64_t bytes) = 0;
    virtual bool Sync() = 0;
    virtual ~CpraImpl() {}
};

}  // namespace CPRA
