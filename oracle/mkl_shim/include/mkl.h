/* Project-written stand-in for <mkl.h> as included by the reference's
 * include/CPRA_Impl.hpp:7-9.  Declares the DFTI and service subsets and the
 * four CBLAS level-1 routines the reference calls
 * (include/detail/MKL_Impl.inl:43,47,61,65).  Test infrastructure only. */
#pragma once
#include "mkl_dfti.h"
#include "mkl_service.h"

typedef int MKL_INT;

/* y = a*x + b*y on complex vectors (a, b point to one complex scalar) */
void cblas_caxpby(MKL_INT n, const void* a, const void* x, MKL_INT incx,
                  const void* b, void* y, MKL_INT incy);
void cblas_zaxpby(MKL_INT n, const void* a, const void* x, MKL_INT incx,
                  const void* b, void* y, MKL_INT incy);
/* x = a*x on complex vectors */
void cblas_cscal(MKL_INT n, const void* a, void* x, MKL_INT incx);
void cblas_zscal(MKL_INT n, const void* a, void* x, MKL_INT incx);
