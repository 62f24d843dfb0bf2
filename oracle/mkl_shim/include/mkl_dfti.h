/* Project-written stand-in for the subset of Intel oneMKL 2024.1 DFTI that the
 * reference operator backend calls (include/MKL_Impl.hpp:24-120,
 * include/detail/MKL_Impl.inl:132-171).  oneMKL is not installed here; this
 * header lets the reference's own MklImpl<T> source compile unchanged so it can
 * serve as the parity oracle.  Test infrastructure only.
 *
 * Semantics restated from the published DFTI interface: complex-to-complex,
 * in-place, batched (DFTI_NUMBER_OF_TRANSFORMS, DFTI_INPUT_DISTANCE), forward
 * transform unscaled, backward transform multiplied by DFTI_BACKWARD_SCALE.
 * Only rank 1 and rank 2 descriptors are accepted: the reference builds its
 * rank-3 descriptor from a 2-element length array (MKL_Impl.hpp:46-47), which
 * would read past the array, so rank 3 is refused with an error status. */
#pragma once
#include <cstdint>

typedef long MKL_LONG;

enum DFTI_CONFIG_VALUE {
    DFTI_SINGLE = 35,
    DFTI_DOUBLE = 36,
    DFTI_COMPLEX = 32,
    DFTI_REAL = 33,
};

enum DFTI_CONFIG_PARAM {
    DFTI_FORWARD_SCALE = 4,
    DFTI_BACKWARD_SCALE = 5,
    DFTI_NUMBER_OF_TRANSFORMS = 7,
    DFTI_INPUT_DISTANCE = 14,
    DFTI_OUTPUT_DISTANCE = 15,
};

#define DFTI_NO_ERROR 0
#define DFTI_INVALID_CONFIGURATION 2
#define DFTI_BAD_DESCRIPTOR 5
#define DFTI_UNIMPLEMENTED 6

struct CpraShimDftiDesc;
typedef CpraShimDftiDesc* DFTI_DESCRIPTOR_HANDLE;

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* handle, DFTI_CONFIG_VALUE precision,
                              DFTI_CONFIG_VALUE domain, MKL_LONG rank, const MKL_LONG* lengths);
/* rank-1 overload: the published macro accepts a scalar length for rank 1 */
MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* handle, DFTI_CONFIG_VALUE precision,
                              DFTI_CONFIG_VALUE domain, MKL_LONG rank, MKL_LONG length);
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE handle, DFTI_CONFIG_PARAM param, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE handle);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE handle, void* inout);
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE handle, void* inout);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE* handle);
MKL_LONG DftiErrorClass(MKL_LONG status, MKL_LONG error_class);
char* DftiErrorMessage(MKL_LONG status);
