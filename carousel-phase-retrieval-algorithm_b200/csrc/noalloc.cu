// ConvergeError without any allocation: cpra_b200_converge_error_noalloc.
//
// Some callers cannot allocate GPU memory while they run:
//  * a process whose device memory is already reserved by another allocator
//    (a framework's caching allocator, a fixed memory pool), where a raw
//    cudaMalloc fails even though the pool has room;
//  * a loop that must not stall other streams: cudaFree synchronises the whole
//    device;
//  * a run that must not fail halfway through on an out-of-memory error.
// The regular entry point allocates its reduction buffers on first use in a
// context, and creating a context allocates too.  This one needs no context
// and uses a fixed scratch array compiled into the library instead.
//
// The scratch is a file-scope static __device__ array of
// CPRA_B200_NOALLOC_MAX_BATCH * (2 * CONVERGE_BLOCKS + 1) doubles (264 KiB for
// 256 members): every GPU that loads the library holds it until the process
// exits.  Its device address is looked up once per device, on the first call
// made with that device current.  CUDA loads a library's device code lazily,
// so that first call is also when the array itself is placed in device
// memory: make it at start-up, before a memory pool reserves the device and
// before any stream capture, and later calls allocate nothing.  The address
// stays valid for the life of the device's primary context; do not use the
// entry point across cudaDeviceReset.  All calls share the array: the partial
// sums are written in full by every call before they are read, so nothing has
// to start at zero, but two calls that overlap on the GPU (on different
// streams, or from different host threads) race on it.
#include "cpra_b200.h"
#include "cpra_internal.h"

#include <cmath>
#include <mutex>
#include <string>

namespace cpra_b200 {
namespace {

constexpr uint64_t kMaxBatch = CPRA_B200_NOALLOC_MAX_BATCH;
constexpr uint64_t kPartials = kMaxBatch * CONVERGE_BLOCKS * 2;  // doubles
constexpr uint64_t kSums = kMaxBatch * 2;                        // doubles
constexpr uint64_t kErr = kMaxBatch;                             // one double per member

static __device__ __align__(256) double g_noalloc_scratch[kPartials + kSums + kErr];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

int fail(int code, const std::string& m) {
    set_last_error(m);
    return code;
}

// err[i] = sqrt(sum |old_i|^2) / sqrt(sum |new_i|^2), the division the regular
// entry point performs on the host, rounded to T once
template <typename T>
__global__ void k_err_from_sums(const double* __restrict__ sums, T* __restrict__ err, uint64_t batch) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < batch; i += (uint64_t)gridDim.x * blockDim.x)
        err[i] = (T)(sqrt(sums[2 * i]) / sqrt(sums[2 * i + 1]));
}

// device address of the scratch array for the current device (looked up once)
int scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(CPRA_B200_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(CPRA_B200_EUNSUP, "converge_error_noalloc: device index above 63");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(CPRA_B200_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CPRA_B200_OK;
}

}  // namespace
}  // namespace cpra_b200

using namespace cpra_b200;

extern "C" int cpra_b200_converge_error_noalloc(int dtype, void* flat_old, const void* flat_new, void* err_host,
                                                uint64_t m, uint64_t n, uint64_t l, uint64_t batch_size,
                                                void* stream) {
    if (dtype != CPRA_B200_F32 && dtype != CPRA_B200_F64)
        return fail(CPRA_B200_EARG, "converge_error_noalloc: dtype must be F32 or F64");
    if (!flat_old || !flat_new || !err_host) return fail(CPRA_B200_EARG, "converge_error_noalloc: null pointer");
    if (m == 0 || n == 0 || l == 0 || batch_size == 0)
        return fail(CPRA_B200_EARG, "converge_error_noalloc: zero size");
    if (batch_size > kMaxBatch)
        return fail(CPRA_B200_EARG, "converge_error_noalloc: batch_size " + std::to_string(batch_size) +
                                        " exceeds the static scratch limit of " + std::to_string(kMaxBatch) +
                                        " members (use cpra_b200_converge_error)");
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    const bool dbl = (dtype == CPRA_B200_F64);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* partials = scratch;
    double* sums = scratch + kPartials;
    double* errd = scratch + kPartials + kSums;
    // CUDA_Impl.inl:155: old <- 1*new + (-1)*old, then the two norms per member
    cudaError_t e = launch_merge_add(dbl, flat_new, flat_old, 1.0, -1.0, m * n * l * batch_size, st);
    if (e == cudaSuccess) e = launch_norm_pairs(dbl, flat_old, flat_new, m * n, m * n * l, batch_size, partials, sums, st);
    if (e == cudaSuccess) {
        if (dbl)
            k_err_from_sums<double><<<1, 256, 0, st>>>(sums, errd, batch_size);
        else
            k_err_from_sums<float><<<1, 256, 0, st>>>(sums, reinterpret_cast<float*>(errd), batch_size);
        count_launches();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(err_host, errd, batch_size * (dbl ? sizeof(double) : sizeof(float)), cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(CPRA_B200_ECUDA, std::string("converge_error_noalloc: ") + cudaGetErrorName(e) + " (" +
                                         cudaGetErrorString(e) + ")");
    return CPRA_B200_OK;
}
