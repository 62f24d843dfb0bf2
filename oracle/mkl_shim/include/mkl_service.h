/* Project-written stand-in for oneMKL's service functions used by the
 * reference (include/Allocator.hpp:56-70): 64-byte aligned allocation.
 * Test infrastructure only. */
#pragma once
#include <cstddef>

void* mkl_malloc(size_t bytes, int alignment);
void mkl_free(void* ptr);
