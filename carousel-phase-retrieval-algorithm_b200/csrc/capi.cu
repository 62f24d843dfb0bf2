// C-ABI of the B200 backend (include/cpra_b200.h): context, argument checks,
// and the call recorder that turns the reference driver's per-operator
// difference-map iterations into fused launches.
//
// Recorder.  The reference drivers issue each difference-map iteration as 12
// operator calls (src/CPRA_MKL.cpp:94-110).  A context holds back a
// Forward2D and the calls that follow it while they still form a prefix of
// that pattern; when all 12 have arrived it holds the whole iteration, and
// further identical iterations only increment a counter.  Anything else
// (another operator, Memcpy, Sync, ConvergeError, a call that breaks the
// pattern) first launches what is held -- the fused kernel for whole
// iterations, the per-operator kernels for a partial prefix -- and then runs
// normally.  Program order is preserved, so results are the per-operator
// results; the fused kernel performs the same arithmetic.
#include "cpra_b200.h"
#include "cpra_internal.h"
#include "angle_table.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <mutex>
#include <string>
#include <functional>
#include <thread>
#include <vector>

using namespace cpra_b200;

namespace cpra_b200 {

static std::atomic<uint64_t> g_launches{0};
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int sm_count() {
    static std::mutex mu;
    static std::map<int, int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
    return n;
}

}  // namespace cpra_b200

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace

void cpra_b200::set_last_error(const std::string& msg) { g_last_error = msg; }

namespace {

int cuda_fail(cudaError_t e, const char* where) {
    return fail(CPRA_B200_ECUDA, std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define CPRA_CHECK_CUDA(expr, where)                   \
    do {                                               \
        cudaError_t _e = (expr);                       \
        if (_e != cudaSuccess) return cuda_fail(_e, where); \
    } while (0)

enum class OpKind { Fwd2D, Bwd2D, DataReal, Merge, Space, Fwd3D, Bwd3D };

struct Op {
    OpKind kind;
    void* dst;        // operand modified in place
    const void* src;  // constraint plane or merge source
    uint64_t num, batch;
    double alpha, beta;
};

struct DmPattern {
    void *x, *t1, *t2;
    const void *A, *S;
    uint64_t num, batch;
    DmCoef c;
    int dim = 2;  // 2: Forward2D/Backward2D iteration; 3: the same with Forward3D/Backward3D
    bool operator==(const DmPattern& o) const {
        return dim == o.dim && x == o.x && t1 == o.t1 && t2 == o.t2 && A == o.A && S == o.S && num == o.num &&
               batch == o.batch &&
               c.a1 == o.c.a1 && c.b1 == o.c.b1 && c.a2 == o.c.a2 && c.b2 == o.c.b2 && c.a3 == o.c.a3 &&
               c.b3 == o.c.b3 && c.a4 == o.c.a4 && c.b4 == o.c.b4;
    }
};

// exp(-2 pi i t / L) for t < L, long double, exact on the quadrant points
template <typename T>
std::vector<T> twiddle_table(uint64_t L) {
    std::vector<T> w(2 * L);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (uint64_t t = 0; t < L; ++t) {
        long double c, s;
        if ((4 * t) % L == 0) {
            const int q = (int)((4 * t) / L);
            const long double cq[4] = {1.0L, 0.0L, -1.0L, 0.0L};
            const long double sq[4] = {0.0L, 1.0L, 0.0L, -1.0L};
            c = cq[q];
            s = sq[q];
        } else {
            const long double a = 2.0L * pi * (long double)t / (long double)L;
            c = cosl(a);
            s = sinl(a);
        }
        w[2 * t] = (T)c;
        w[2 * t + 1] = (T)(-s);
    }
    return w;
}

}  // namespace

struct GraphEntry {
    std::string key;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;
    uint64_t epoch = 0;
};

struct BucketLane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    void* scratch = nullptr;
    uint64_t scratch_bytes = 0;
};

// A stream of the carousel driver's wavefront schedule with its own t1, t2,
// old (drv, 3 planes of the batch) and work scratch; ev[p] marks angle p of
// the lane's latest episode done.  Lane 0 is the context's own stream and
// buffers.
struct RunLane {
    cudaStream_t stream = nullptr;
    void* drv = nullptr;
    uint64_t drv_bytes = 0;
    void* work = nullptr;
    uint64_t work_bytes = 0;
    std::vector<cudaEvent_t> ev;
    cudaEvent_t join = nullptr;
};

struct cpra_b200_ctx {
    bool dbl = false;
    uint64_t m = 1, n = 1, l = 1, batch = 1;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::map<uint64_t, void*> tw;  // length -> device table
    void* work = nullptr;
    uint64_t work_bytes = 0;
    double* partials = nullptr;
    double* sums = nullptr;
    double* host_sums = nullptr;
    uint64_t red_cap = 0;  // batch members the reduction buffers hold
    bool fusion = true;
    int space_mode = SPACE_THRESHOLD;
    int data_mode = DATA_SKIP_ZERO;
    uint64_t seed = 0x5eedull;
    uint64_t init_calls = 0;
    std::vector<Op> pending;
    DmPattern held{};
    int held_iters = 0;
    int deferred_error = CPRA_B200_OK;
    std::string deferred_msg;
    // opt-in timing of fused launches
    bool timing = false;
    std::vector<cudaEvent_t> free_events;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timed;
    uint64_t timed_pattern_iters = 0;
    // driver-level buffers of cpra_b200_cpra_run: t1, t2, old (batch planes each)
    void* drv = nullptr;
    uint64_t drv_bytes = 0;
    double* err_sums = nullptr;
    double* host_err = nullptr;
    uint64_t err_cap = 0;
    // shrinkwrap blur tables per (side, updates, sigma_start, sigma_end)
    std::map<std::tuple<uint64_t, int, double, double>, void*> blur_cache;
    // streams, join events and scratch of cpra_b200_hio_batched's buckets
    std::vector<BucketLane> bucket_streams;
    cudaEvent_t fork_event = nullptr;
    // CUDA graphs of cpra_run / hio_batched calls (CPRA_B200_OPT_GRAPH): one
    // per distinct argument set, valid while no context buffer has moved
    // cpra_b200_refine: gV, Adam moments, per-step losses; cpra_b200_best_start: sums
    void* refine_buf = nullptr;
    uint64_t refine_bytes = 0;
    void* best_sums = nullptr;
    uint64_t best_bytes = 0;
    // raw-file I/O: two pinned staging chunks (CPRA_B200_OPT_IO_CHUNK bytes
    // each), their events, and cpra_b200_cpra_files' device buffers (A, S,
    // the starts, the gathered real parts)
    void* io_pinned[2] = {nullptr, nullptr};
    uint64_t io_pinned_bytes = 0;
    cudaEvent_t io_ev[2] = {nullptr, nullptr};
    cudaEvent_t io_ready = nullptr;
    uint64_t io_chunk = 64ull << 20;
    void* io_dev = nullptr;
    uint64_t io_dev_bytes = 0;
    void* io_A = nullptr;
    uint64_t io_A_bytes = 0;
    void* io_S = nullptr;
    uint64_t io_S_bytes = 0;
    void* io_x = nullptr;
    uint64_t io_x_bytes = 0;
    // cpra_b200_cpra_run's lanes (CPRA_B200_OPT_LANES: 0 automatic)
    std::vector<RunLane> run_lanes;
    cudaEvent_t lane_fork = nullptr;
    int lanes_opt = 0;
    // CPRA_B200_OPT_AUTOTUNE: measured lane counts per run key, and the
    // choice of the last cpra_b200_cpra_run that used the cache (0: none)
    bool autotune = false;
    std::vector<std::pair<std::string, int>> tune_cache;
    int tuned_lanes = 0;
    // cpra_b200_cpra_run_host: device copies of x, A, S, the copy stream and events
    void* hx = nullptr;
    uint64_t hx_bytes = 0;
    void* hA = nullptr;
    uint64_t hA_bytes = 0;
    void* hS = nullptr;
    uint64_t hS_bytes = 0;
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> run_events;
    // slices sorted by direction for the gathers over slices (angle_table.cuh)
    void* atab = nullptr;
    uint64_t atab_bytes = 0;
    // the slice operator's per-slice orientation table (sines and cosines)
    void* otab = nullptr;
    uint64_t otab_bytes = 0;
    bool graphs = false;
    bool capturing = false;
    uint64_t epoch = 0;  // bumped whenever a context buffer is freed or reallocated
    std::vector<GraphEntry> graph_cache;
    // patterns per chunk of the large-plane HIO passes (0: the whole batch)
    uint64_t hio_chunk = 0;
    // CPRA_B200_OPT_TMEM: the 128 x 128 fused kernels keep their iterates in tensor memory
    bool tmem = true;
    // CPRA_B200_OPT_FUSED3D: the 3D loops as fused axis passes (off: the operator kernels)
    bool fused3d = false;
    // CPRA_B200_OPT_HIO_CLUSTER: CTAs per pattern of the cluster HIO kernel (0 off, 1 automatic)
    int hio_cluster = 1;
    int hio_cluster_trial = -1;  // >= 0: the size under measurement by the tuner
    std::vector<std::pair<int, int>> cluster_active;  // (side * 100 + size, resident clusters)
    int sm_count = 0;
    // device word a cluster kernel sets when a wait for a peer CTA's data ran
    // out; once such a kernel was launched (directly or in a captured graph),
    // every Sync reads it (and clears it when set)
    int* dev_err = nullptr;
    bool err_pending = false;
    // CPRA_B200_OPT_FAILURE_TEST: the next cluster HIO launch withholds one
    // CTA's first blocks (its peers' waits run out)
    bool failure_test = false;

    size_t esize() const { return dbl ? sizeof(double) : sizeof(float); }
    size_t csize() const { return 2 * esize(); }
    uint64_t plane() const { return m * n; }
    double round_t(double v) const { return dbl ? v : (double)(float)v; }
};

namespace {

const void* twiddles(cpra_b200_ctx* c, uint64_t L) {
    auto it = c->tw.find(L);
    return it == c->tw.end() ? nullptr : it->second;
}

int ensure_twiddles(cpra_b200_ctx* c, uint64_t L) {
    if (L < 1 || c->tw.count(L)) return CPRA_B200_OK;
    void* d = nullptr;
    const size_t bytes = 2 * L * c->esize();
    CPRA_CHECK_CUDA(cudaMalloc(&d, bytes), "cudaMalloc(twiddles)");
    cudaError_t e;
    if (c->dbl) {
        auto h = twiddle_table<double>(L);
        e = cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice);
    } else {
        auto h = twiddle_table<float>(L);
        e = cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_fail(e, "cudaMemcpy(twiddles)");
    }
    c->tw[L] = d;
    return CPRA_B200_OK;
}

int ensure_work(cpra_b200_ctx* c, uint64_t bytes) {
    if (c->work_bytes >= bytes) return CPRA_B200_OK;
    ++c->epoch;
    if (c->work) {
        cudaStreamSynchronize(c->stream);
        cudaFree(c->work);
        c->work = nullptr;
        c->work_bytes = 0;
    }
    CPRA_CHECK_CUDA(cudaMalloc(&c->work, bytes), "cudaMalloc(work)");
    c->work_bytes = bytes;
    return CPRA_B200_OK;
}

int ensure_reduction(cpra_b200_ctx* c, uint64_t members) {
    if (c->red_cap >= members) return CPRA_B200_OK;
    ++c->epoch;
    if (c->partials) {
        cudaStreamSynchronize(c->stream);
        cudaFree(c->partials);
        cudaFree(c->sums);
        cudaFreeHost(c->host_sums);
        c->partials = c->sums = c->host_sums = nullptr;
        c->red_cap = 0;
    }
    CPRA_CHECK_CUDA(cudaMalloc(&c->partials, sizeof(double) * 2 * CONVERGE_BLOCKS * members), "cudaMalloc(partials)");
    CPRA_CHECK_CUDA(cudaMalloc(&c->sums, sizeof(double) * 2 * members), "cudaMalloc(sums)");
    CPRA_CHECK_CUDA(cudaMallocHost(&c->host_sums, sizeof(double) * 2 * members), "cudaMallocHost(sums)");
    c->red_cap = members;
    return CPRA_B200_OK;
}

int ensure_buffer(cpra_b200_ctx* c, void** buf, uint64_t* have, uint64_t bytes, const char* what) {
    if (*have >= bytes) return CPRA_B200_OK;
    ++c->epoch;
    if (*buf) {
        cudaDeviceSynchronize();
        cudaFree(*buf);
        *buf = nullptr;
        *have = 0;
    }
    CPRA_CHECK_CUDA(cudaMalloc(buf, bytes), what);
    *have = bytes;
    return CPRA_B200_OK;
}

bool overlap(const void* a, uint64_t abytes, const void* b, uint64_t bbytes) {
    const char* pa = static_cast<const char*>(a);
    const char* pb = static_cast<const char*>(b);
    return pa < pb + bbytes && pb < pa + abytes;
}

// ---- per-operator execution ---------------------------------------------------
int run_fft2d(cpra_b200_ctx* c, void* x, bool inverse) {
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n))
        return fail(CPRA_B200_EUNSUP, "2D transform: each size must be 1 or even and at most 4096");
    const bool pow2 = ((c->m & (c->m - 1)) == 0) && ((c->n & (c->n - 1)) == 0) && c->m <= 1024 && c->n <= 1024;
    if (!pow2) {
        int r = ensure_work(c, c->batch * c->plane() * c->csize());
        if (r) return r;
    }
    // DFTI_BACKWARD_SCALE = (T)1.0 / (m*n) (include/MKL_Impl.hpp:40)
    const double scale = c->dbl ? 1.0 / (double)(c->m * c->n) : (double)(1.0f / (float)(c->m * c->n));
    CPRA_CHECK_CUDA(launch_fft2d(c->dbl, x, c->m, c->n, c->batch, inverse, scale, twiddles(c, c->m),
                                 twiddles(c, c->n), c->work, c->stream),
                    inverse ? "Backward2D" : "Forward2D");
    return CPRA_B200_OK;
}

// the 3D transform itself (arguments checked, recorder already flushed)
int exec_fft3d(cpra_b200_ctx* c, void* x, bool inverse) {
    auto p2 = [](uint64_t v) { return (v & (v - 1)) == 0 && v <= 1024; };
    if (!(p2(c->m) && p2(c->n) && p2(c->l))) {
        int r = ensure_work(c, c->batch * c->m * c->n * c->l * c->csize());
        if (r) return r;
    }
    // DFTI_BACKWARD_SCALE = (T)1.0 / (m*n*l) (include/MKL_Impl.hpp:62)
    const uint64_t vol = c->m * c->n * c->l;
    const double scale = c->dbl ? 1.0 / (double)vol : (double)(1.0f / (float)vol);
    CPRA_CHECK_CUDA(launch_fft3d(c->dbl, x, c->m, c->n, c->l, c->batch, inverse, scale, twiddles(c, c->m),
                                 twiddles(c, c->n), twiddles(c, c->l), c->work, c->stream),
                    inverse ? "Backward3D" : "Forward3D");
    return CPRA_B200_OK;
}

int exec_op(cpra_b200_ctx* c, const Op& op) {
    switch (op.kind) {
        case OpKind::Fwd2D: return run_fft2d(c, op.dst, false);
        case OpKind::Bwd2D: return run_fft2d(c, op.dst, true);
        case OpKind::Fwd3D: return exec_fft3d(c, op.dst, false);
        case OpKind::Bwd3D: return exec_fft3d(c, op.dst, true);
        case OpKind::DataReal:
            CPRA_CHECK_CUDA(launch_data_constraint_real(c->dbl, op.dst, op.src, op.num, op.num / op.batch, c->data_mode,
                                                        c->stream),
                            "DataConstraint");
            return CPRA_B200_OK;
        case OpKind::Space:
            CPRA_CHECK_CUDA(launch_space_constraint(c->dbl, op.dst, op.src, op.num, op.num / op.batch, c->space_mode,
                                                    c->stream),
                            "SpaceConstraint");
            return CPRA_B200_OK;
        case OpKind::Merge:
            CPRA_CHECK_CUDA(launch_merge_add(c->dbl, op.src, op.dst, op.alpha, op.beta, op.num, c->stream),
                            "MergeAddData");
            return CPRA_B200_OK;
    }
    return fail(CPRA_B200_EARG, "unknown operator");
}

// fused difference-map iterations on either path: one CTA per pattern up to
// 128 x 128, line passes through the work buffer at 256 and 512
bool dm_fusable(const cpra_b200_ctx* c) {
    return dm_fused_supported(c->dbl, c->m, c->n) || dm_large_supported(c->dbl, c->m, c->n, c->space_mode);
}

int run_dm(cpra_b200_ctx* c, const DmArgs& a, const char* what) {
    if (dm_fused_supported(c->dbl, a.M, a.N)) {
        CPRA_CHECK_CUDA(launch_dm_iterations(c->dbl, a, twiddles(c, a.M), c->stream), what);
        return CPRA_B200_OK;
    }
    int r = ensure_work(c, dm_large_scratch_bytes(a.M, a.N, a.batch, a.s_stride));
    if (r) return r;
    CPRA_CHECK_CUDA(launch_dm_large(a, twiddles(c, a.M), c->work, c->stream), what);
    return CPRA_B200_OK;
}

int launch_fused(cpra_b200_ctx* c, const DmPattern& p, int iters, int mix = MIX_NONE, const void* xprev = nullptr,
                 const void* xnext = nullptr, int init_from_x = 0) {
    DmArgs a;
    a.mix = mix;
    a.xprev = xprev;
    a.xnext = xnext;
    a.init_from_x = init_from_x;
    a.x = p.x;
    a.t1 = p.t1;
    a.t2 = p.t2;
    a.A = p.A;
    a.a_stride = 0;
    a.S = p.S;
    a.s_stride = 0;
    a.M = c->m;
    a.N = c->n;
    a.batch = c->batch;
    a.iters = iters;
    a.space_mode = c->space_mode;
    a.data_mode = c->data_mode;
    a.tmem = c->tmem ? 1 : 0;
    a.c = p.c;
    a.L = (p.dim == 3) ? c->l : 1;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    const bool timed = c->timing && !c->capturing;  // graph replays are not timed per launch
    if (timed) {
        for (cudaEvent_t& e : ev) {
            if (!c->free_events.empty()) {
                e = c->free_events.back();
                c->free_events.pop_back();
            } else {
                CPRA_CHECK_CUDA(cudaEventCreate(&e), "cudaEventCreate");
            }
        }
        CPRA_CHECK_CUDA(cudaEventRecord(ev[0], c->stream), "cudaEventRecord");
    }
    int r;
    if (p.dim == 3) {
        const uint64_t vol = c->m * c->n * c->l;
        const double scale = c->dbl ? 1.0 / (double)vol : (double)(1.0f / (float)vol);
        CPRA_CHECK_CUDA(launch_dm3d_iterations(c->dbl, a, scale, twiddles(c, c->m), twiddles(c, c->n),
                                               twiddles(c, c->l), c->work, c->stream),
                        "fused 3D difference-map iteration");
        r = CPRA_B200_OK;
    } else {
        r = run_dm(c, a, "fused difference-map iteration");
    }
    if (r) return r;
    if (timed) {
        CPRA_CHECK_CUDA(cudaEventRecord(ev[1], c->stream), "cudaEventRecord");
        c->timed.emplace_back(ev[0], ev[1]);
        c->timed_pattern_iters += c->batch * (uint64_t)iters;
    }
    return CPRA_B200_OK;
}

// `iters` iterations of pattern p: fused when the shape allows, else per call
int dm_any(cpra_b200_ctx* c, const DmPattern& p, int iters) {
    if (iters <= 0) return CPRA_B200_OK;
    if (dm_fusable(c)) return launch_fused(c, p, iters);
    const uint64_t num = p.num;
    const uint64_t B = p.batch;
    for (int i = 0; i < iters; ++i) {
        const Op seq[12] = {
            {OpKind::Fwd2D, p.t1, nullptr, 0, 0, 0, 0},   {OpKind::DataReal, p.t1, p.A, num, B, 0, 0},
            {OpKind::Bwd2D, p.t1, nullptr, 0, 0, 0, 0},   {OpKind::Merge, p.t1, p.x, num, 1, p.c.a1, p.c.b1},
            {OpKind::Space, p.t1, p.S, num, B, 0, 0},     {OpKind::Space, p.t2, p.S, num, B, 0, 0},
            {OpKind::Merge, p.t2, p.x, num, 1, p.c.a2, p.c.b2}, {OpKind::Fwd2D, p.t2, nullptr, 0, 0, 0, 0},
            {OpKind::DataReal, p.t2, p.A, num, B, 0, 0},  {OpKind::Bwd2D, p.t2, nullptr, 0, 0, 0, 0},
            {OpKind::Merge, p.x, p.t1, num, 1, p.c.a3, p.c.b3}, {OpKind::Merge, p.x, p.t2, num, 1, p.c.a4, p.c.b4}};
        for (const Op& op : seq) {
            int r = exec_op(c, op);
            if (r) return r;
        }
    }
    return CPRA_B200_OK;
}

// launch everything held, in program order
int flush(cpra_b200_ctx* c) {
    int rc = CPRA_B200_OK;
    if (c->held_iters > 0) {
        rc = launch_fused(c, c->held, c->held_iters);
        c->held_iters = 0;
    }
    std::vector<Op> ops;
    ops.swap(c->pending);
    for (const Op& op : ops) {
        int r = exec_op(c, op);
        if (r && !rc) rc = r;
    }
    if (rc && !c->deferred_error) {
        c->deferred_error = rc;
        c->deferred_msg = g_last_error;
    }
    return rc;
}

// surface an error from a launch that was deferred by the recorder
int take_deferred(cpra_b200_ctx* c) {
    if (!c->deferred_error) return CPRA_B200_OK;
    int rc = c->deferred_error;
    c->deferred_error = CPRA_B200_OK;
    return fail(rc, "deferred launch failed: " + c->deferred_msg);
}

bool fusable_shape(const cpra_b200_ctx* c) { return c->fusion && dm_fusable(c); }
// the 3D iteration fuses for power-of-two volumes (axis passes)
bool fusable_shape3d(const cpra_b200_ctx* c) {
    return c->fusion && c->fused3d && c->l > 1 && constraint3d_fused_supported(c->m, c->n, c->l);
}

// Does `op` extend the pending prefix (of length k) of the pattern?
bool extends(const cpra_b200_ctx* c, const Op& op) {
    const std::vector<Op>& P = c->pending;
    const size_t k = P.size();
    const bool d3 = P[0].kind == OpKind::Fwd3D;
    const uint64_t plane = c->plane() * (d3 ? c->l : 1);  // the constraints' plane (num / batch)
    const uint64_t num = plane * c->batch;
    const uint64_t cbytes = num * c->csize();
    const uint64_t rbytes = plane * c->esize();
    const OpKind FWD = d3 ? OpKind::Fwd3D : OpKind::Fwd2D, BWD = d3 ? OpKind::Bwd3D : OpKind::Bwd2D;
    auto T1 = [&]() { return P[0].dst; };
    auto is_ew = [&](OpKind kind) {
        return op.kind == kind && op.num == num && op.batch == c->batch && op.num % op.batch == 0 &&
               op.num / op.batch == plane;
    };
    switch (k) {
        case 1:  // DataConstraint(t1, A)
            return is_ew(OpKind::DataReal) && op.dst == T1() && !overlap(op.src, rbytes, T1(), cbytes);
        case 2:  // Backward2D(t1)
            return op.kind == BWD && op.dst == T1();
        case 3:  // MergeAddData(x, t1, a1, b1)
            return op.kind == OpKind::Merge && op.num == num && op.dst == T1() && !overlap(op.src, cbytes, T1(), cbytes) &&
                   !overlap(op.src, cbytes, P[1].src, rbytes);
        case 4:  // SpaceConstraint(t1, S)
            return is_ew(OpKind::Space) && op.dst == T1() && !overlap(op.src, rbytes, T1(), cbytes) &&
                   !overlap(op.src, rbytes, P[3].src, cbytes);
        case 5: {  // SpaceConstraint(t2, S)
            const void* X = P[3].src;
            return is_ew(OpKind::Space) && op.src == P[4].src && !overlap(op.dst, cbytes, T1(), cbytes) &&
                   !overlap(op.dst, cbytes, X, cbytes) && !overlap(op.dst, cbytes, P[1].src, rbytes) &&
                   !overlap(op.dst, cbytes, P[4].src, rbytes);
        }
        case 6:  // MergeAddData(x, t2, a2, b2)
            return op.kind == OpKind::Merge && op.num == num && op.src == P[3].src && op.dst == P[5].dst;
        case 7:  // Forward2D(t2)
            return op.kind == FWD && op.dst == P[5].dst;
        case 8:  // DataConstraint(t2, A)
            return is_ew(OpKind::DataReal) && op.dst == P[5].dst && op.src == P[1].src;
        case 9:  // Backward2D(t2)
            return op.kind == BWD && op.dst == P[5].dst;
        case 10:  // MergeAddData(t1, x, a3, b3)
            return op.kind == OpKind::Merge && op.num == num && op.src == T1() && op.dst == P[3].src;
        case 11:  // MergeAddData(t2, x, a4, b4)
            return op.kind == OpKind::Merge && op.num == num && op.src == P[5].dst && op.dst == P[3].src;
        default: return false;
    }
}

DmPattern pattern_of(const std::vector<Op>& P) {
    DmPattern d;
    d.t1 = P[0].dst;
    d.A = P[1].src;
    d.x = const_cast<void*>(P[3].src);
    d.S = P[4].src;
    d.t2 = P[5].dst;
    d.num = P[1].num;
    d.batch = P[1].batch;
    d.c = {P[3].alpha, P[3].beta, P[6].alpha, P[6].beta, P[10].alpha, P[10].beta, P[11].alpha, P[11].beta};
    d.dim = (P[0].kind == OpKind::Fwd3D) ? 3 : 2;
    return d;
}

// Entry for every operator that the recorder may hold.
int submit(cpra_b200_ctx* c, const Op& op) {
    if (c->pending.empty()) {
        const bool start2 = op.kind == OpKind::Fwd2D && fusable_shape(c);
        const bool start3 = op.kind == OpKind::Fwd3D && fusable_shape3d(c);
        if (start2 || start3) {
            if (c->held_iters > 0 && (op.dst != c->held.t1 || c->held.dim != (start3 ? 3 : 2))) {
                int r = flush(c);
                if (r) return take_deferred(c);
            }
            c->pending.push_back(op);
            return take_deferred(c);
        }
        int r = flush(c);
        if (r) return take_deferred(c);
        return exec_op(c, op);
    }
    if (extends(c, op)) {
        c->pending.push_back(op);
        if (c->pending.size() == 12) {
            DmPattern p = pattern_of(c->pending);
            c->pending.clear();
            if (c->held_iters > 0 && p == c->held) {
                ++c->held_iters;
            } else {
                if (c->held_iters > 0) {
                    int r = launch_fused(c, c->held, c->held_iters);
                    c->held_iters = 0;
                    if (r) return r;
                }
                c->held = p;
                c->held_iters = 1;
            }
        }
        return take_deferred(c);
    }
    int r = flush(c);
    if (r) return take_deferred(c);
    return submit(c, op);
}

int check_ctx(cpra_b200_ctx* c) {
    if (!c) return fail(CPRA_B200_EARG, "null context");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return CPRA_B200_OK;
}

#define CTX_OR_RETURN(c)            \
    do {                            \
        int _r = check_ctx(c);      \
        if (_r) return _r;          \
    } while (0)

}  // namespace

extern "C" {

const char* cpra_b200_last_error(void) { return g_last_error.c_str(); }

uint64_t cpra_b200_kernels_launched(void) { return g_launches.load(std::memory_order_relaxed); }

int cpra_b200_create(cpra_b200_ctx** out, int dtype, uint64_t m, uint64_t n, uint64_t l, uint64_t batch_size) {
    if (!out) return fail(CPRA_B200_EARG, "null output pointer");
    *out = nullptr;
    if (dtype != CPRA_B200_F32 && dtype != CPRA_B200_F64) return fail(CPRA_B200_EARG, "dtype must be F32 or F64");
    if (m == 0 || n == 0 || l == 0 || batch_size == 0) return fail(CPRA_B200_EARG, "sizes must be positive");
    auto* c = new cpra_b200_ctx();
    c->dbl = (dtype == CPRA_B200_F64);
    c->m = m;
    c->n = n;
    c->l = l;
    c->batch = batch_size;
    cudaError_t e = cudaGetDevice(&c->device);
    if (e == cudaSuccess) e = cudaStreamCreate(&c->stream);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cudaStreamCreate");
    }
    e = cudaMalloc(reinterpret_cast<void**>(&c->dev_err), sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->dev_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        cpra_b200_destroy(c);
        return cuda_fail(e, "cudaMalloc(error word)");
    }
    for (uint64_t L : {m, n, l}) {
        if (L <= 4096) {
            int r = ensure_twiddles(c, L);
            if (r) {
                cpra_b200_destroy(c);
                return r;
            }
        }
    }
    *out = c;
    return CPRA_B200_OK;
}

int cpra_b200_destroy(cpra_b200_ctx* c) {
    if (!c) return CPRA_B200_OK;
    cudaSetDevice(c->device);
    int rc = flush(c);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& kv : c->tw) cudaFree(kv.second);
    if (c->dev_err) cudaFree(c->dev_err);
    if (c->work) cudaFree(c->work);
    if (c->partials) cudaFree(c->partials);
    if (c->sums) cudaFree(c->sums);
    if (c->host_sums) cudaFreeHost(c->host_sums);
    if (c->drv) cudaFree(c->drv);
    for (auto& kv : c->blur_cache) cudaFree(kv.second);
    for (BucketLane& lane : c->bucket_streams) {
        if (lane.stream) cudaStreamSynchronize(lane.stream);
        if (lane.scratch) cudaFree(lane.scratch);
        if (lane.done) cudaEventDestroy(lane.done);
        if (lane.stream) cudaStreamDestroy(lane.stream);
    }
    if (c->fork_event) cudaEventDestroy(c->fork_event);
    for (GraphEntry& g : c->graph_cache) cudaGraphExecDestroy(g.exec);
    if (c->refine_buf) cudaFree(c->refine_buf);
    if (c->best_sums) cudaFree(c->best_sums);
    if (c->atab) cudaFree(c->atab);
    if (c->otab) cudaFree(c->otab);
    for (RunLane& lane : c->run_lanes) {
        if (lane.stream) cudaStreamSynchronize(lane.stream);
        if (lane.drv) cudaFree(lane.drv);
        if (lane.work) cudaFree(lane.work);
        for (cudaEvent_t e : lane.ev) cudaEventDestroy(e);
        if (lane.join) cudaEventDestroy(lane.join);
        if (lane.stream) cudaStreamDestroy(lane.stream);
    }
    if (c->lane_fork) cudaEventDestroy(c->lane_fork);
    for (int k = 0; k < 2; ++k) {
        if (c->io_pinned[k]) cudaFreeHost(c->io_pinned[k]);
        if (c->io_ev[k]) cudaEventDestroy(c->io_ev[k]);
    }
    if (c->io_ready) cudaEventDestroy(c->io_ready);
    for (void* b : {c->io_dev, c->io_A, c->io_S, c->io_x})
        if (b) cudaFree(b);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    if (c->hx) cudaFree(c->hx);
    if (c->hA) cudaFree(c->hA);
    if (c->hS) cudaFree(c->hS);
    for (cudaEvent_t e : c->run_events) cudaEventDestroy(e);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->err_sums) cudaFree(c->err_sums);
    if (c->host_err) cudaFreeHost(c->host_err);
    for (auto& pr : c->timed) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    for (cudaEvent_t e : c->free_events) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return rc;
}

int cpra_b200_set_option(cpra_b200_ctx* c, int option, int64_t value) {
    CTX_OR_RETURN(c);
    int r = flush(c);
    if (r) return take_deferred(c);
    switch (option) {
        case CPRA_B200_OPT_FUSION: c->fusion = value != 0; break;
        case CPRA_B200_OPT_SPACE_MODE:
            if (value != SPACE_THRESHOLD && value != SPACE_POSITIVE_SCALED) return fail(CPRA_B200_EARG, "space mode");
            c->space_mode = (int)value;
            break;
        case CPRA_B200_OPT_DATA_MODE:
            if (value != DATA_SKIP_ZERO && value != DATA_ALWAYS) return fail(CPRA_B200_EARG, "data mode");
            c->data_mode = (int)value;
            break;
        case CPRA_B200_OPT_SEED: c->seed = (uint64_t)value; c->init_calls = 0; break;
        case CPRA_B200_OPT_KERNEL_TIMING: c->timing = value != 0; break;
        case CPRA_B200_OPT_GRAPH:
            c->graphs = value != 0;
            if (!c->graphs) {
                for (GraphEntry& g : c->graph_cache) cudaGraphExecDestroy(g.exec);
                c->graph_cache.clear();
            }
            break;
        case CPRA_B200_OPT_HIO_CHUNK:
            if (value < 0) return fail(CPRA_B200_EARG, "hio chunk must be >= 0");
            c->hio_chunk = (uint64_t)value;
            break;
        case CPRA_B200_OPT_LANES:
            if (value < 0 || value > CPRA_B200_MAX_LANES) return fail(CPRA_B200_EARG, "lanes must be 0..16");
            c->lanes_opt = (int)value;
            break;
        case CPRA_B200_OPT_IO_CHUNK:
            if (value < 4096) return fail(CPRA_B200_EARG, "io chunk must be >= 4096 bytes");
            c->io_chunk = (uint64_t)value;
            break;
        case CPRA_B200_OPT_AUTOTUNE: c->autotune = value != 0; break;
        case CPRA_B200_OPT_TMEM: c->tmem = value != 0; break;
        case CPRA_B200_OPT_FUSED3D: c->fused3d = value != 0; break;
        case CPRA_B200_OPT_HIO_CLUSTER:
            if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 16)
                return fail(CPRA_B200_EARG, "hio cluster must be 0, 1, 2, 4, 8 or 16");
            c->hio_cluster = (int)value;
            break;
        case CPRA_B200_OPT_FAILURE_TEST: c->failure_test = value != 0; break;
        default: return fail(CPRA_B200_EARG, "unknown option");
    }
    return CPRA_B200_OK;
}

int cpra_b200_get_stream(cpra_b200_ctx* c, void** stream) {
    CTX_OR_RETURN(c);
    if (!stream) return fail(CPRA_B200_EARG, "null output pointer");
    *stream = (void*)c->stream;
    return CPRA_B200_OK;
}

int cpra_b200_alloc(cpra_b200_ctx* c, void** out, uint64_t bytes, int managed) {
    CTX_OR_RETURN(c);
    if (!out) return fail(CPRA_B200_EARG, "null output pointer");
    *out = nullptr;
    if (bytes == 0) return fail(CPRA_B200_EARG, "zero-byte allocation");
    if (managed)
        CPRA_CHECK_CUDA(cudaMallocManaged(out, bytes, cudaMemAttachGlobal), "cudaMallocManaged");
    else
        CPRA_CHECK_CUDA(cudaMalloc(out, bytes), "cudaMalloc");
    return CPRA_B200_OK;
}

int cpra_b200_free(cpra_b200_ctx* c, void* ptr) {
    CTX_OR_RETURN(c);
    int r = flush(c);
    if (r) return take_deferred(c);
    if (ptr) CPRA_CHECK_CUDA(cudaFree(ptr), "cudaFree");
    return CPRA_B200_OK;
}

int cpra_b200_initialize(cpra_b200_ctx* c, void* flat, uint64_t num) {
    CTX_OR_RETURN(c);
    if (num < 1) return fail(CPRA_B200_EARG, "Initialize: num < 1");  // MKL_Impl.inl:11
    if (!flat) return fail(CPRA_B200_EARG, "Initialize: null pointer");
    int r = flush(c);
    if (r) return take_deferred(c);
    CPRA_CHECK_CUDA(launch_uniform(c->dbl, flat, num, c->seed, c->init_calls++, c->stream), "Initialize");
    return CPRA_B200_OK;
}

int cpra_b200_forward2d(cpra_b200_ctx* c, void* x) {
    CTX_OR_RETURN(c);
    if (!x) return fail(CPRA_B200_EARG, "Forward2D: null pointer");
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n))
        return fail(CPRA_B200_EUNSUP, "Forward2D: each size must be 1 or even and at most 4096");
    return submit(c, Op{OpKind::Fwd2D, x, nullptr, 0, 0, 0, 0});
}

int cpra_b200_backward2d(cpra_b200_ctx* c, void* x) {
    CTX_OR_RETURN(c);
    if (!x) return fail(CPRA_B200_EARG, "Backward2D: null pointer");
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n))
        return fail(CPRA_B200_EUNSUP, "Backward2D: each size must be 1 or even and at most 4096");
    return submit(c, Op{OpKind::Bwd2D, x, nullptr, 0, 0, 0, 0});
}

static bool shift_size_ok(uint64_t v) { return v == 1 || (v % 2) == 0; }

int cpra_b200_fftshift2d(cpra_b200_ctx* c, void* x, uint64_t M, uint64_t N, uint64_t B) {
    CTX_OR_RETURN(c);
    if (!x) return fail(CPRA_B200_EARG, "FFTShift2D: null pointer");
    if (!shift_size_ok(M) || !shift_size_ok(N))
        return fail(CPRA_B200_EARG, "FFTShift2D: sizes must be even (or 1); the reference swap is a shift only then");
    int r = flush(c);
    if (r) return take_deferred(c);
    CPRA_CHECK_CUDA(launch_fftshift2d(c->dbl, x, M, N, B, c->stream), "FFTShift2D");
    return CPRA_B200_OK;
}

static int run_fft3d(cpra_b200_ctx* c, void* x, bool inverse) {
    if (!x) return fail(CPRA_B200_EARG, inverse ? "Backward3D: null pointer" : "Forward3D: null pointer");
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n) || !fft_length_supported(c->l))
        return fail(CPRA_B200_EUNSUP, "3D transform: each size must be 1 or even and at most 4096");
    return submit(c, Op{inverse ? OpKind::Bwd3D : OpKind::Fwd3D, x, nullptr, 0, 0, 0, 0});
}

namespace {

// CPRA_B200_OPT_AUTOTUNE for choices that leave the results unchanged: the
// cached choice of `key`, or, for a new key, a measurement: each candidate
// runs once untimed and once timed, prepare() restoring the trial inputs
// before each run and run(k) enqueuing candidate k; the fastest is cached.
int tuned_choice(cpra_b200_ctx* c, const std::string& key, const std::vector<uint64_t>& cand,
                 const std::function<int()>& prepare, const std::function<int(uint64_t)>& run, uint64_t* out) {
    for (const auto& e : c->tune_cache)
        if (e.first == key) {
            *out = (uint64_t)e.second;
            return CPRA_B200_OK;
        }
    struct Events {
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~Events() {
            for (cudaEvent_t v : e)
                if (v) cudaEventDestroy(v);
        }
    } ev;
    CPRA_CHECK_CUDA(cudaEventCreate(&ev.e[0]), "cudaEventCreate");
    CPRA_CHECK_CUDA(cudaEventCreate(&ev.e[1]), "cudaEventCreate");
    std::vector<float> ms(cand.size(), 0.0f);
    for (int pass = 0; pass < 2; ++pass) {
        for (size_t k = 0; k < cand.size(); ++k) {
            int r = prepare();
            if (r) return r;
            CPRA_CHECK_CUDA(cudaEventRecord(ev.e[0], c->stream), "autotune");
            r = run(cand[k]);
            if (r) return r;
            CPRA_CHECK_CUDA(cudaEventRecord(ev.e[1], c->stream), "autotune");
            CPRA_CHECK_CUDA(cudaEventSynchronize(ev.e[1]), "autotune");
            CPRA_CHECK_CUDA(cudaEventElapsedTime(&ms[k], ev.e[0], ev.e[1]), "autotune");
        }
    }
    size_t best = 0;
    for (size_t k = 1; k < cand.size(); ++k)
        if (ms[k] < ms[best]) best = k;
    c->tune_cache.emplace_back(key, (int)cand[best]);
    *out = cand[best];
    return CPRA_B200_OK;
}

// a stream capture is under way on the context's stream (ours or the caller's)
bool stream_capturing(cpra_b200_ctx* c) {
    if (c->capturing) return true;
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(c->stream, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone;
}

// a device buffer for the duration of a measurement (freed on scope exit)
struct TrialBuffer {
    cpra_b200_ctx* c;
    void* p = nullptr;
    explicit TrialBuffer(cpra_b200_ctx* ctx) : c(ctx) {}
    bool alloc(uint64_t bytes) {
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();  // out of memory is not sticky
            p = nullptr;
            return false;
        }
        return true;
    }
    ~TrialBuffer() {
        if (p) {
            cudaStreamSynchronize(c->stream);
            cudaFree(p);
        }
    }
};

// `iters` repetitions of the benchmark's 3D step, as fused axis passes or as
// the four operator kernels (the same bits)
int constraint3d_path(cpra_b200_ctx* c, void* x, const void* C, const void* S, int iters, bool fused, double scale) {
    const uint64_t vol = c->m * c->n * c->l, num = vol * c->batch;
    if (fused) {
        CPRA_CHECK_CUDA(launch_constraint3d(c->dbl, x, C, S, c->m, c->n, c->l, c->batch, iters, c->space_mode, scale,
                                            twiddles(c, c->m), twiddles(c, c->n), twiddles(c, c->l), c->work,
                                            c->stream),
                        "constraint3d");
        return CPRA_B200_OK;
    }
    int r = ensure_work(c, num * c->csize());
    if (r) return r;
    for (int it = 0; it < iters; ++it) {
        CPRA_CHECK_CUDA(launch_fft3d(c->dbl, x, c->m, c->n, c->l, c->batch, false, scale, twiddles(c, c->m),
                                     twiddles(c, c->n), twiddles(c, c->l), c->work, c->stream),
                        "constraint3d");
        CPRA_CHECK_CUDA(launch_data_constraint_complex(c->dbl, x, C, num, vol, c->stream), "constraint3d");
        CPRA_CHECK_CUDA(launch_fft3d(c->dbl, x, c->m, c->n, c->l, c->batch, true, scale, twiddles(c, c->m),
                                     twiddles(c, c->n), twiddles(c, c->l), c->work, c->stream),
                        "constraint3d");
        CPRA_CHECK_CUDA(launch_space_constraint(c->dbl, x, S, num, vol, c->space_mode, c->stream), "constraint3d");
    }
    return CPRA_B200_OK;
}

}  // namespace

int cpra_b200_constraint3d(cpra_b200_ctx* c, void* x, const void* C, const void* S, int iters) {
    CTX_OR_RETURN(c);
    if (!x || !C || !S) return fail(CPRA_B200_EARG, "constraint3d: null pointer");
    if (iters < 0) return fail(CPRA_B200_EARG, "constraint3d: iters must be >= 0");
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n) || !fft_length_supported(c->l))
        return fail(CPRA_B200_EUNSUP, "constraint3d: each size must be 1 or even and at most 4096");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t vol = c->m * c->n * c->l, num = vol * c->batch;
    // DFTI_BACKWARD_SCALE = (T)1.0 / (m*n*l) (include/MKL_Impl.hpp:62)
    const double scale = c->dbl ? 1.0 / (double)vol : (double)(1.0f / (float)vol);
    const bool can_fuse = constraint3d_fused_supported(c->m, c->n, c->l);
    bool fused = c->fused3d && can_fuse;
    // CPRA_B200_OPT_AUTOTUNE: the faster of the two paths, measured once per
    // shape on a copy of x (one iteration each)
    if (c->autotune && can_fuse && iters > 0 && !stream_capturing(c)) {
        TrialBuffer trial(c);
        if (trial.alloc(num * c->csize())) {
            const std::string key = "constraint3d:" + std::to_string(c->m) + "," + std::to_string(c->n) + "," +
                                    std::to_string(c->l) + "," + std::to_string(c->batch) + "," +
                                    std::to_string(c->dbl) + "," + std::to_string(c->space_mode);
            uint64_t choice = fused ? 1 : 0;
            r = tuned_choice(
                c, key, {0, 1},
                [&]() -> int {
                    CPRA_CHECK_CUDA(cudaMemcpyAsync(trial.p, x, num * c->csize(), cudaMemcpyDeviceToDevice, c->stream),
                                    "autotune");
                    return CPRA_B200_OK;
                },
                [&](uint64_t k) { return constraint3d_path(c, trial.p, C, S, 1, k != 0, scale); }, &choice);
            if (r) return r;
            fused = choice != 0;
        }
    }
    return constraint3d_path(c, x, C, S, iters, fused, scale);
}

int cpra_b200_forward3d(cpra_b200_ctx* c, void* x) {
    CTX_OR_RETURN(c);
    return run_fft3d(c, x, false);
}

int cpra_b200_backward3d(cpra_b200_ctx* c, void* x) {
    CTX_OR_RETURN(c);
    return run_fft3d(c, x, true);
}

int cpra_b200_fftshift3d(cpra_b200_ctx* c, void* x, uint64_t M, uint64_t N, uint64_t L, uint64_t B) {
    CTX_OR_RETURN(c);
    if (!x) return fail(CPRA_B200_EARG, "FFTShift3D: null pointer");
    if (!shift_size_ok(M) || !shift_size_ok(N) || !shift_size_ok(L))
        return fail(CPRA_B200_EARG, "FFTShift3D: sizes must be even (or 1)");
    int r = flush(c);
    if (r) return take_deferred(c);
    CPRA_CHECK_CUDA(launch_fftshift3d(c->dbl, x, M, N, L, B, c->stream), "FFTShift3D");
    return CPRA_B200_OK;
}

static int ew_args(const char* what, const void* x, const void* k, uint64_t num, uint64_t batch) {
    // MKL_Impl.inl:73,89,112: num == 0 or batch_size == 0 -> false
    if (num == 0 || batch == 0) return fail(CPRA_B200_EARG, std::string(what) + ": num and batch_size must be positive");
    if (num / batch == 0) return fail(CPRA_B200_EARG, std::string(what) + ": num < batch_size (empty plane)");
    if (!x || !k) return fail(CPRA_B200_EARG, std::string(what) + ": null pointer");
    return CPRA_B200_OK;
}

int cpra_b200_space_constraint(cpra_b200_ctx* c, void* x, const void* s, uint64_t num, uint64_t batch) {
    CTX_OR_RETURN(c);
    int r = ew_args("SpaceConstraint", x, s, num, batch);
    if (r) return r;
    return submit(c, Op{OpKind::Space, x, s, num, batch, 0, 0});
}

int cpra_b200_data_constraint_real(cpra_b200_ctx* c, void* x, const void* a, uint64_t num, uint64_t batch) {
    CTX_OR_RETURN(c);
    int r = ew_args("DataConstraint", x, a, num, batch);
    if (r) return r;
    return submit(c, Op{OpKind::DataReal, x, a, num, batch, 0, 0});
}

int cpra_b200_data_constraint_complex(cpra_b200_ctx* c, void* x, const void* k, uint64_t num, uint64_t batch) {
    CTX_OR_RETURN(c);
    int r = ew_args("DataConstraint(complex)", x, k, num, batch);
    if (r) return r;
    r = flush(c);
    if (r) return take_deferred(c);
    CPRA_CHECK_CUDA(launch_data_constraint_complex(c->dbl, x, k, num, num / batch, c->stream), "DataConstraint(complex)");
    return CPRA_B200_OK;
}

int cpra_b200_merge_add(cpra_b200_ctx* c, const void* src, void* dst, double alpha, double beta, uint64_t num) {
    CTX_OR_RETURN(c);
    const double a = c->round_t(alpha), b = c->round_t(beta);
    // MKL_Impl.inl:34: alpha == 0 or num == 0 -> false
    if (a == 0.0 || num == 0) return fail(CPRA_B200_EARG, "MergeAddData: alpha == 0 or num == 0");
    if (!src || !dst) return fail(CPRA_B200_EARG, "MergeAddData: null pointer");
    return submit(c, Op{OpKind::Merge, dst, src, num, 1, a, b});
}

int cpra_b200_normalization(cpra_b200_ctx* c, void* x, double norm, uint64_t num) {
    CTX_OR_RETURN(c);
    const double nt = c->round_t(norm);
    // MKL_Impl.inl:55: norm == 0 or num == 0 -> false
    if (nt == 0.0 || num == 0) return fail(CPRA_B200_EARG, "Normalization: norm == 0 or num == 0");
    if (!x) return fail(CPRA_B200_EARG, "Normalization: null pointer");
    int r = flush(c);
    if (r) return take_deferred(c);
    // MKL_Impl.inl:57-58: scal by T(1.0 / norm)
    CPRA_CHECK_CUDA(launch_scale(c->dbl, x, c->round_t(1.0 / nt), num, c->stream), "Normalization");
    return CPRA_B200_OK;
}

int cpra_b200_real2d_to_3d(cpra_b200_ctx* c, const void* src, void* dst, const void* angles, uint64_t m, uint64_t n,
                           uint64_t p, uint64_t l) {
    CTX_OR_RETURN(c);
    if (!src || !dst || !angles) return fail(CPRA_B200_EARG, "Real2DTo3DInterpolation: null pointer");
    if (m == 0 || n == 0 || p == 0 || l == 0) return fail(CPRA_B200_EARG, "Real2DTo3DInterpolation: zero size");
    int r = flush(c);
    if (r) return take_deferred(c);
    CPRA_CHECK_CUDA(launch_real2d_to_3d(c->dbl, src, dst, angles, m, n, p, l, c->stream), "Real2DTo3DInterpolation");
    return CPRA_B200_OK;
}

int cpra_b200_complex2d_to_3d(cpra_b200_ctx* c, const void* src, void* dst, const void* angles, uint64_t m,
                              uint64_t n, uint64_t p, uint64_t l) {
    CTX_OR_RETURN(c);
    if (!src || !dst || !angles) return fail(CPRA_B200_EARG, "Complex2DTo3DInterpolation: null pointer");
    if (m == 0 || n == 0 || p == 0 || l == 0) return fail(CPRA_B200_EARG, "Complex2DTo3DInterpolation: zero size");
    int r = flush(c);
    if (r) return take_deferred(c);
    void* atab = nullptr;
    if (p <= (uint64_t)ANGLE_TABLE_MAX) {
        int rr = ensure_buffer(c, &c->atab, &c->atab_bytes, angle_table_bytes(p), "cudaMalloc(angle table)");
        if (rr) return rr;
        atab = c->atab;
    }
    CPRA_CHECK_CUDA(launch_complex2d_to_3d(c->dbl, src, dst, angles, m, n, p, l, atab, c->stream),
                    "Complex2DTo3DInterpolation");
    return CPRA_B200_OK;
}

int cpra_b200_converge_error(cpra_b200_ctx* c, void* old_, const void* new_, void* err_host, uint64_t m, uint64_t n,
                             uint64_t l, uint64_t batch) {
    CTX_OR_RETURN(c);
    if (!old_ || !new_ || !err_host) return fail(CPRA_B200_EARG, "ConvergeError: null pointer");
    if (m == 0 || n == 0 || l == 0 || batch == 0) return fail(CPRA_B200_EARG, "ConvergeError: zero size");
    if (batch > 65535) return fail(CPRA_B200_EUNSUP, "ConvergeError: batch_size above 65535");
    int r = flush(c);
    if (r) return take_deferred(c);
    r = ensure_reduction(c, batch);
    if (r) return r;
    // CUDA_Impl.inl:155: old <- 1*new + (-1)*old
    CPRA_CHECK_CUDA(launch_merge_add(c->dbl, new_, old_, 1.0, -1.0, m * n * l * batch, c->stream), "ConvergeError");
    CPRA_CHECK_CUDA(launch_norm_pairs(c->dbl, old_, new_, m * n, m * n * l, batch, c->partials, c->sums, c->stream),
                    "ConvergeError");
    CPRA_CHECK_CUDA(cudaMemcpyAsync(c->host_sums, c->sums, sizeof(double) * 2 * batch, cudaMemcpyDeviceToHost, c->stream),
                    "ConvergeError");
    CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "ConvergeError");
    for (uint64_t i = 0; i < batch; ++i) {
        const double e = std::sqrt(c->host_sums[2 * i]) / std::sqrt(c->host_sums[2 * i + 1]);
        if (c->dbl)
            static_cast<double*>(err_host)[i] = e;
        else
            static_cast<float*>(err_host)[i] = (float)e;
    }
    return CPRA_B200_OK;
}

int cpra_b200_memcpy(cpra_b200_ctx* c, void* dst, const void* src, uint64_t bytes) {
    CTX_OR_RETURN(c);
    if ((!dst || !src) && bytes) return fail(CPRA_B200_EARG, "Memcpy: null pointer");
    int r = flush(c);
    if (r) return take_deferred(c);
    if (bytes) CPRA_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream), "Memcpy");
    return CPRA_B200_OK;
}

int cpra_b200_sync(cpra_b200_ctx* c) {
    CTX_OR_RETURN(c);
    int r = flush(c);
    if (r) return take_deferred(c);
    CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "Sync");
    if (c->err_pending) {
        int h = 0;
        CPRA_CHECK_CUDA(cudaMemcpy(&h, c->dev_err, sizeof(int), cudaMemcpyDeviceToHost), "Sync");
        if (h) {
            CPRA_CHECK_CUDA(cudaMemset(c->dev_err, 0, sizeof(int)), "Sync");
            return fail(CPRA_B200_ECUDA,
                        "hio cluster kernel: a CTA's wait for its peers' data ran out; the results are invalid");
        }
    }
    return CPRA_B200_OK;
}

int cpra_b200_dm_iterations(cpra_b200_ctx* c, void* x, void* t1, void* t2, const void* A, uint64_t a_stride,
                            const void* S, uint64_t s_stride, uint64_t batch, double beta, int iters) {
    CTX_OR_RETURN(c);
    if (!x || !t1 || !t2 || !A || !S) return fail(CPRA_B200_EARG, "dm_iterations: null pointer");
    if (batch == 0 || iters < 0) return fail(CPRA_B200_EARG, "dm_iterations: batch must be positive, iters >= 0");
    const double b = c->round_t(beta);
    if (b == 0.0) return fail(CPRA_B200_EARG, "dm_iterations: beta == 0");
    if (!dm_fusable(c))
        return fail(CPRA_B200_EUNSUP,
                    "dm_iterations: fused path needs float and square 32, 64, 128 planes, or 256 and 512 with the "
                    "threshold SpaceConstraint");
    if (!dm_fused_supported(c->dbl, c->m, c->n) && s_stride != 0 && s_stride != c->plane())
        return fail(CPRA_B200_EARG, "dm_iterations: at 256 and 512 s_stride must be 0 or m*n");
    int r = flush(c);
    if (r) return take_deferred(c);
    if (iters == 0) return CPRA_B200_OK;
    // src/CPRA_MKL.cpp:98,103,109,110: coefficients in double from a T beta, passed as T
    DmArgs a;
    a.x = x;
    a.t1 = t1;
    a.t2 = t2;
    a.A = A;
    a.a_stride = a_stride;
    a.S = S;
    a.s_stride = s_stride;
    a.M = c->m;
    a.N = c->n;
    a.batch = batch;
    a.iters = iters;
    a.space_mode = c->space_mode;
    a.data_mode = c->data_mode;
    a.tmem = c->tmem ? 1 : 0;
    a.c = {c->round_t(-1.0 / b), c->round_t(1.0 + 1.0 / b), c->round_t(1.0 / b), c->round_t(1.0 - 1.0 / b),
           c->round_t(b),        1.0,                         c->round_t(-1.0 * b), 1.0};
    return run_dm(c, a, "dm_iterations");
}

int cpra_b200_rfactor(cpra_b200_ctx* c, const void* x, const void* A, uint64_t a_stride, uint64_t batch,
                      double* r_host) {
    CTX_OR_RETURN(c);
    if (!x || !A || !r_host) return fail(CPRA_B200_EARG, "rfactor: null pointer");
    if (batch == 0) return fail(CPRA_B200_EARG, "rfactor: batch must be positive");
    if (batch > 65535) return fail(CPRA_B200_EUNSUP, "rfactor: batch above 65535");
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n))
        return fail(CPRA_B200_EUNSUP, "rfactor: each plane size must be 1 or even and at most 4096");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t plane = c->plane();
    // the spectra go to a work buffer (the input stays untouched); the
    // non-power-of-two transform path needs a second one of the same size
    const uint64_t bytes = batch * plane * c->csize();
    r = ensure_work(c, 2 * bytes);
    if (r) return r;
    r = ensure_reduction(c, batch);
    if (r) return r;
    char* F = static_cast<char*>(c->work);
    CPRA_CHECK_CUDA(cudaMemcpyAsync(F, x, bytes, cudaMemcpyDefault, c->stream), "rfactor");
    CPRA_CHECK_CUDA(launch_fft2d(c->dbl, F, c->m, c->n, batch, false, 1.0, twiddles(c, c->m), twiddles(c, c->n),
                                 F + bytes, c->stream),
                    "rfactor");
    CPRA_CHECK_CUDA(launch_rfactor_sums(c->dbl, F, A, a_stride, plane, batch, c->partials, c->sums, c->stream),
                    "rfactor");
    CPRA_CHECK_CUDA(cudaMemcpyAsync(c->host_sums, c->sums, sizeof(double) * 2 * batch, cudaMemcpyDeviceToHost, c->stream),
                    "rfactor");
    CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "rfactor");
    for (uint64_t i = 0; i < batch; ++i) r_host[i] = c->host_sums[2 * i] / c->host_sums[2 * i + 1];
    return CPRA_B200_OK;
}

namespace {

// Device tables of the shrinkwrap blur: for update k of `updates`, sigma moves
// linearly from s0 to s1; entry i of a table is the DFT of a normalised
// periodic Gaussian (real and even) at the frequency (i + L/2) mod L that the
// sign-modulated transform puts at index i.  Cached per (L, updates, s0, s1).
int blur_tables(cpra_b200_ctx* c, uint64_t L, int updates, double s0, double s1, const void** out) {
    const auto key = std::make_tuple(L, updates, s0, s1);
    auto it = c->blur_cache.find(key);
    if (it != c->blur_cache.end()) {
        *out = it->second;
        return CPRA_B200_OK;
    }
    std::vector<double> cs(L);
    for (uint64_t ph = 0; ph < L; ++ph) cs[ph] = std::cos(2.0 * 3.141592653589793238462643383279502884 * (double)ph / (double)L);
    std::vector<float> tab((size_t)updates * L);
    std::vector<double> g(L);
    for (int k = 0; k < updates; ++k) {
        const double sg = updates > 1 ? s0 + (s1 - s0) * k / (updates - 1) : s0;
        double sum = 0.0;
        for (uint64_t n = 0; n < L; ++n) {
            const double d = (double)std::min<uint64_t>(n, L - n);
            g[n] = std::exp(-d * d / (2.0 * sg * sg));
            sum += g[n];
        }
        for (uint64_t f = 0; f < L; ++f) {
            const uint64_t fu = (f + L / 2) % L;
            double acc = 0.0;
            for (uint64_t n = 0; n < L; ++n) acc += g[n] * cs[(n * fu) % L];
            tab[(size_t)k * L + f] = (float)(acc / sum);
        }
    }
    void* d = nullptr;
    const size_t bytes = tab.size() * sizeof(float);
    CPRA_CHECK_CUDA(cudaMalloc(&d, bytes), "cudaMalloc(blur tables)");
    const cudaError_t e = cudaMemcpy(d, tab.data(), bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_fail(e, "cudaMemcpy(blur tables)");
    }
    c->blur_cache[key] = d;
    *out = d;
    return CPRA_B200_OK;
}

struct HioJob {
    uint64_t L, batch;
    void* x;
    const void* A;
    uint64_t a_stride;
    void* S;
    uint64_t s_stride;
    void* estimate;
};
struct HioParams {
    int iters, sw_every, positivity;
    double beta, sigma_start, sigma_end, threshold;
    int updates() const { return sw_every > 0 ? iters / sw_every : 0; }
};

bool hio_side_supported(bool dbl, uint64_t L) {
    return hio_fused_supported(dbl, L, L) || hio_large_supported(dbl, L, L);
}

// scratch bytes of one job: Y, V, the support mask and the maxima of a chunk
uint64_t hio_scratch_bytes(bool dbl, uint64_t L, uint64_t chunk) {
    if (hio_fused_supported(dbl, L, L)) return 0;
    return chunk * L * L * 8 + chunk * L * L * 4 + chunk * L * L / 8 + chunk * 4;
}

// clusters of `cluster` CTAs of the side-L kernel resident at once (cached)
int cluster_resident(cpra_b200_ctx* c, uint64_t L, int cluster) {
    const int key = (int)L * 100 + cluster;
    for (const auto& e : c->cluster_active)
        if (e.first == key) return e.second;
    const int n = hio_cluster_max_active(L, cluster);
    c->cluster_active.emplace_back(key, n);
    return n;
}

// CTAs per pattern of the cluster kernel for a job of `batch` patterns of
// side L, or 0 for the one-CTA kernels (32-128) and the line passes (256, 512).
// Automatic: the cluster kernel only where the batch cannot fill the device
// otherwise, the largest cluster whose CTAs take one SM each and all fit at
// once (128: 8, 4 or 2; 256: 8); at 128 only with the tensor-memory kernel
// as the alternative, whose bits it shares.  A batch that fills the SMs with
// one CTA per pattern (128) or runs as line passes (256) is faster without.
int hio_cluster_for(cpra_b200_ctx* c, uint64_t L, uint64_t batch) {
    if (c->dbl || batch == 0) return 0;
    if (c->hio_cluster_trial >= 0) return c->hio_cluster_trial;
    if (c->hio_cluster == 0) return 0;
    if (c->hio_cluster > 1) return hio_cluster_supported(c->dbl, L, c->hio_cluster) ? c->hio_cluster : 0;
    if (L == 128 && !c->tmem) return 0;
    if (c->sm_count == 0 && cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess)
        return 0;
    for (int cl : {8, 4, 2}) {
        if (!hio_cluster_supported(c->dbl, L, cl)) continue;
        if (batch * (uint64_t)cl <= (uint64_t)c->sm_count && batch <= (uint64_t)cluster_resident(c, L, cl)) return cl;
    }
    return 0;
}

// scratch of a job: none for the fused and cluster kernels
uint64_t hio_job_scratch(cpra_b200_ctx* c, uint64_t L, uint64_t batch, uint64_t chunk) {
    return hio_cluster_for(c, L, batch) ? 0 : hio_scratch_bytes(c->dbl, L, chunk);
}

// enqueue one job on `st` (arguments already checked); `scratch` holds
// hio_scratch_bytes(L, chunk)
int hio_enqueue(cpra_b200_ctx* c, const HioJob& j, const HioParams& h, uint64_t chunk, void* scratch,
                cudaStream_t st) {
    const int updates = h.updates();
    HioArgs a;
    a.x = j.x;
    a.estimate = j.estimate;
    a.A = j.A;
    a.a_stride = j.a_stride;
    a.S = j.S;
    a.s_stride = j.s_stride;
    a.blur = nullptr;
    if (updates > 0) {
        int r = blur_tables(c, j.L, updates, h.sigma_start, h.sigma_end, &a.blur);
        if (r) return r;
    }
    a.M = a.N = j.L;
    a.batch = j.batch;
    a.iters = h.iters;
    a.sw_every = updates > 0 ? h.sw_every : 0;
    a.positivity = h.positivity ? 1 : 0;
    a.data_mode = c->data_mode;
    a.tmem = c->tmem ? 1 : 0;
    a.beta = c->round_t(h.beta);
    a.threshold = h.threshold;
    int r = ensure_twiddles(c, j.L);
    if (r) return r;
    if (const int cl = hio_cluster_for(c, j.L, j.batch)) {
        a.err = c->dev_err;
        a.withhold = c->failure_test ? 1 : 0;
        c->failure_test = false;
        c->err_pending = true;
        CPRA_CHECK_CUDA(launch_hio_cluster(a, cl, twiddles(c, j.L), st), "hio_shrinkwrap");
        return CPRA_B200_OK;
    }
    if (hio_fused_supported(c->dbl, j.L, j.L)) {
        CPRA_CHECK_CUDA(launch_hio_iterations(c->dbl, a, twiddles(c, j.L), st), "hio_shrinkwrap");
        return CPRA_B200_OK;
    }
    const uint64_t plane = j.L * j.L;
    char* w = static_cast<char*>(scratch);
    const uint64_t yb = chunk * plane * 8, vb = chunk * plane * 4, mb = chunk * plane / 8;  // multiples of 256
    CPRA_CHECK_CUDA(launch_hio_large(a, twiddles(c, j.L), w, w + yb, reinterpret_cast<unsigned int*>(w + yb + vb + mb),
                                     reinterpret_cast<uint32_t*>(w + yb + vb), chunk, st),
                    "hio_shrinkwrap");
    return CPRA_B200_OK;
}

extern "C++" {
// Runs `enqueue` (stream work only: no allocation, no synchronisation) on the
// context's stream, or, with CPRA_B200_OPT_GRAPH on, replays the CUDA graph
// captured from it for the same key, capturing it on the first call.  A
// graph holds the context buffers' addresses, so it is used only while the
// context's buffer epoch is the one it was captured in.
template <class Fn>
int run_maybe_graph(cpra_b200_ctx* c, const std::string& key, Fn enqueue) {
    if (!c->graphs) return enqueue();
    for (GraphEntry& g : c->graph_cache) {
        if (g.key == key && g.epoch == c->epoch) {
            CPRA_CHECK_CUDA(cudaGraphLaunch(g.exec, c->stream), "cudaGraphLaunch");
            count_launches(g.launches);
            return CPRA_B200_OK;
        }
    }
    const uint64_t n0 = g_launches.load(std::memory_order_relaxed);
    CPRA_CHECK_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
    c->capturing = true;
    const uint64_t epoch0 = c->epoch;
    int r = enqueue();
    c->capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (r || e != cudaSuccess || c->epoch != epoch0) {
        if (graph) cudaGraphDestroy(graph);
        if (r) return r;
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        return fail(CPRA_B200_ECUDA, "graph capture: a context buffer moved during capture");
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
    // the capture counted the graph's kernels once, for this first launch
    const uint64_t launches = g_launches.load(std::memory_order_relaxed) - n0;
    if (c->graph_cache.size() >= 16) {
        cudaGraphExecDestroy(c->graph_cache.front().exec);
        c->graph_cache.erase(c->graph_cache.begin());
    }
    c->graph_cache.push_back(GraphEntry{key, exec, launches, c->epoch});
    CPRA_CHECK_CUDA(cudaGraphLaunch(exec, c->stream), "cudaGraphLaunch");
    return CPRA_B200_OK;
}

// a graph cache key: the raw bytes of the values
template <class... V>
std::string graph_key(const char* tag, const V&... v) {
    std::string k(tag);
    (k.append(reinterpret_cast<const char*>(&v), sizeof(V)), ...);
    return k;
}
}  // extern "C++"

int hio_check_params(const HioParams& h, const char* who) {
    if (h.iters < 0) return fail(CPRA_B200_EARG, std::string(who) + ": iters must be >= 0");
    if (h.updates() > 0 && !(h.sigma_start > 0.0 && h.sigma_end > 0.0))
        return fail(CPRA_B200_EARG, std::string(who) + ": sigma must be positive");
    return CPRA_B200_OK;
}


}  // namespace

int cpra_b200_hio_shrinkwrap(cpra_b200_ctx* c, void* x, const void* A, uint64_t a_stride, void* S, uint64_t s_stride,
                             uint64_t batch, int iters, double beta, int sw_every, double sigma_start,
                             double sigma_end, double threshold, int positivity, void* estimate) {
    CTX_OR_RETURN(c);
    if (!x || !A || !S) return fail(CPRA_B200_EARG, "hio_shrinkwrap: null pointer");
    if (batch == 0 || iters < 0) return fail(CPRA_B200_EARG, "hio_shrinkwrap: batch must be positive, iters >= 0");
    if (c->m != c->n || !hio_side_supported(c->dbl, c->m))
        return fail(CPRA_B200_EUNSUP, "hio_shrinkwrap: needs float and square 32, 64, 128, 256 or 512 planes");
    const HioParams h{iters, sw_every, positivity, beta, sigma_start, sigma_end, threshold};
    int r = hio_check_params(h, "hio_shrinkwrap");
    if (r) return r;
    if (h.updates() > 0 && s_stride < c->plane())
        return fail(CPRA_B200_EARG, "hio_shrinkwrap: shrinkwrap updates each pattern's support: s_stride >= m*n");
    r = flush(c);
    if (r) return take_deferred(c);
    if (iters == 0 && !estimate) return CPRA_B200_OK;
    uint64_t chunk = (c->hio_chunk == 0) ? batch : std::min(c->hio_chunk, batch);
    // CPRA_B200_OPT_AUTOTUNE (chunk 0 only): the line passes' chunk measured
    // once per (side, batch) among the whole batch, a half and a quarter, on
    // copies of x and S, min(iters, 20) iterations each (the chunk changes
    // the schedule only)
    // CPRA_B200_OPT_AUTOTUNE with the automatic cluster choice at 128 (the
    // tensor-memory kernel): one CTA per pattern against clusters of 2, 4 and
    // 8, measured once per (batch, iterations) on copies of x and S,
    // min(iters, 20) iterations each (all four write the same bits)
    int tuned_cluster = -1;
    if (c->autotune && c->hio_cluster == 1 && !c->dbl && c->m == 128 && c->tmem && iters > 0 && !stream_capturing(c)) {
        const uint64_t plane = c->plane();
        const uint64_t xb = batch * plane * c->csize();
        const uint64_t sb = (s_stride ? batch * s_stride : plane) * c->esize();
        TrialBuffer trial(c);
        if (trial.alloc(xb + sb + 256)) {
            void* tx = trial.p;
            void* tS = static_cast<char*>(trial.p) + (xb + 255) / 256 * 256;
            HioParams ht = h;
            ht.iters = std::min(iters, 20);
            const std::string key = "hio_cluster:" + std::to_string(c->m) + "," + std::to_string(batch) + "," +
                                    std::to_string(ht.iters) + "," + std::to_string(sw_every) + "," +
                                    std::to_string(c->data_mode) + "," + std::to_string(positivity);
            uint64_t pick = 0;
            r = tuned_choice(
                c, key, {0, 2, 4, 8},
                [&]() -> int {
                    CPRA_CHECK_CUDA(cudaMemcpyAsync(tx, x, xb, cudaMemcpyDeviceToDevice, c->stream), "autotune");
                    CPRA_CHECK_CUDA(cudaMemcpyAsync(tS, S, sb, cudaMemcpyDeviceToDevice, c->stream), "autotune");
                    return CPRA_B200_OK;
                },
                [&](uint64_t k) {
                    c->hio_cluster_trial = (int)k;
                    const int rr = hio_enqueue(c, HioJob{c->m, batch, tx, A, a_stride, tS, s_stride, nullptr}, ht, 0,
                                               nullptr, c->stream);
                    c->hio_cluster_trial = -1;
                    return rr;
                },
                &pick);
            if (r) return r;
            tuned_cluster = (int)pick;
        }
    }
    if (c->autotune && c->hio_chunk == 0 && !hio_fused_supported(c->dbl, c->m, c->n) &&
        !hio_cluster_for(c, c->m, batch) && batch > 1 && iters > 0 && !stream_capturing(c)) {
        const uint64_t plane = c->plane();
        const uint64_t xb = batch * plane * c->csize();
        // S too: the passes write the support back (packed at the start, unpacked at the end)
        const uint64_t sb = (s_stride ? batch * s_stride : plane) * c->esize();
        TrialBuffer trial(c);
        r = ensure_work(c, hio_scratch_bytes(c->dbl, c->m, batch));
        if (r) return r;
        if (trial.alloc(xb + sb + 256)) {
            void* tx = trial.p;
            void* tS = static_cast<char*>(trial.p) + (xb + 255) / 256 * 256;
            std::vector<uint64_t> cand;
            for (uint64_t k : {batch, (batch + 1) / 2, (batch + 3) / 4})
                if (std::find(cand.begin(), cand.end(), k) == cand.end()) cand.push_back(k);
            HioParams ht = h;
            ht.iters = std::min(iters, 20);
            const std::string key = "hio_chunk:" + std::to_string(c->m) + "," + std::to_string(batch) + "," +
                                    std::to_string(ht.iters) + "," + std::to_string(sw_every) + "," +
                                    std::to_string(c->data_mode);
            r = tuned_choice(
                c, key, cand,
                [&]() -> int {
                    CPRA_CHECK_CUDA(cudaMemcpyAsync(tx, x, xb, cudaMemcpyDeviceToDevice, c->stream), "autotune");
                    CPRA_CHECK_CUDA(cudaMemcpyAsync(tS, S, sb, cudaMemcpyDeviceToDevice, c->stream), "autotune");
                    return CPRA_B200_OK;
                },
                [&](uint64_t k) {
                    return hio_enqueue(c, HioJob{c->m, batch, tx, A, a_stride, tS, s_stride, nullptr}, ht, k, c->work,
                                       c->stream);
                },
                &chunk);
            if (r) return r;
        }
    }
    r = ensure_work(c, hio_job_scratch(c, c->m, batch, chunk));
    if (r) return r;
    c->hio_cluster_trial = tuned_cluster;
    r = hio_enqueue(c, HioJob{c->m, batch, x, A, a_stride, S, s_stride, estimate}, h, chunk, c->work, c->stream);
    c->hio_cluster_trial = -1;
    return r;
}

int cpra_b200_hio_batched(cpra_b200_ctx* c, const cpra_b200_hio_bucket* buckets, int n_buckets, int iters,
                          double beta, int sw_every, double sigma_start, double sigma_end, double threshold,
                          int positivity) {
    CTX_OR_RETURN(c);
    if (!buckets || n_buckets <= 0) return fail(CPRA_B200_EARG, "hio_batched: no buckets");
    if (n_buckets > CPRA_B200_MAX_BUCKETS) return fail(CPRA_B200_EARG, "hio_batched: too many buckets");
    const HioParams h{iters, sw_every, positivity, beta, sigma_start, sigma_end, threshold};
    int r = hio_check_params(h, "hio_batched");
    if (r) return r;
    for (int i = 0; i < n_buckets; ++i) {
        const cpra_b200_hio_bucket& b = buckets[i];
        if (!b.x || !b.A || !b.S || b.count == 0) return fail(CPRA_B200_EARG, "hio_batched: bucket without data");
        if (!hio_side_supported(c->dbl, b.side))
            return fail(CPRA_B200_EUNSUP, "hio_batched: sides must be 32, 64, 128, 256 or 512 (float context)");
        if ((b.sigma_start > 0.0) != (b.sigma_end > 0.0))
            return fail(CPRA_B200_EARG, "hio_batched: a bucket's sigma_start and sigma_end are both set or neither");
    }
    // each bucket's parameters: its own blur schedule when it has one
    auto bucket_params = [&](const cpra_b200_hio_bucket& b) {
        HioParams hb = h;
        if (b.sigma_start > 0.0) {
            hb.sigma_start = b.sigma_start;
            hb.sigma_end = b.sigma_end;
        }
        return hb;
    };
    r = flush(c);
    if (r) return take_deferred(c);
    if (iters == 0) {
        bool any_estimate = false;
        for (int i = 0; i < n_buckets; ++i) any_estimate |= buckets[i].estimate != nullptr;
        if (!any_estimate) return CPRA_B200_OK;
    }
    // one stream per bucket, forked from and joined back into the context's
    // stream; the most work (pixels x patterns) is enqueued first
    std::vector<int> order(n_buckets);
    for (int i = 0; i < n_buckets; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return buckets[a].side * buckets[a].side * buckets[a].count > buckets[b].side * buckets[b].side * buckets[b].count;
    });
    while ((int)c->bucket_streams.size() < n_buckets) {
        BucketLane lane;
        CPRA_CHECK_CUDA(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        CPRA_CHECK_CUDA(cudaEventCreateWithFlags(&lane.done, cudaEventDisableTiming), "cudaEventCreate");
        c->bucket_streams.push_back(lane);
    }
    if (!c->fork_event) CPRA_CHECK_CUDA(cudaEventCreateWithFlags(&c->fork_event, cudaEventDisableTiming), "cudaEventCreate");
    for (int k = 0; k < n_buckets; ++k) {
        const cpra_b200_hio_bucket& b = buckets[order[k]];
        BucketLane& lane = c->bucket_streams[k];
        const uint64_t chunk = (c->hio_chunk == 0) ? b.count : std::min(c->hio_chunk, b.count);
        r = ensure_buffer(c, &lane.scratch, &lane.scratch_bytes, hio_job_scratch(c, b.side, b.count, chunk),
                          "cudaMalloc(hio_batched scratch)");
        if (r) return r;
        r = ensure_twiddles(c, b.side);
        if (r) return r;
        if (h.updates() > 0) {
            const void* unused;
            const HioParams hb = bucket_params(b);
            r = blur_tables(c, b.side, hb.updates(), hb.sigma_start, hb.sigma_end, &unused);
            if (r) return r;
        }
    }
    auto enqueue = [&]() -> int {
        CPRA_CHECK_CUDA(cudaEventRecord(c->fork_event, c->stream), "hio_batched");
        for (int k = 0; k < n_buckets; ++k) {
            const cpra_b200_hio_bucket& b = buckets[order[k]];
            BucketLane& lane = c->bucket_streams[k];
            const uint64_t plane = b.side * b.side;
            const uint64_t chunk = (c->hio_chunk == 0) ? b.count : std::min(c->hio_chunk, b.count);
            CPRA_CHECK_CUDA(cudaStreamWaitEvent(lane.stream, c->fork_event, 0), "hio_batched");
            int rr = hio_enqueue(c, HioJob{b.side, b.count, b.x, b.A, plane, b.S, plane, b.estimate},
                                 bucket_params(b), chunk, lane.scratch, lane.stream);
            if (rr) return rr;
            CPRA_CHECK_CUDA(cudaEventRecord(lane.done, lane.stream), "hio_batched");
            CPRA_CHECK_CUDA(cudaStreamWaitEvent(c->stream, lane.done, 0), "hio_batched");
        }
        return CPRA_B200_OK;
    };
    std::string key = graph_key("hio_batched", n_buckets, iters, beta, sw_every, sigma_start, sigma_end, threshold,
                                positivity, c->hio_chunk, c->data_mode, c->tmem, c->hio_cluster);
    for (int i = 0; i < n_buckets; ++i) key.append(reinterpret_cast<const char*>(&buckets[i]), sizeof(buckets[i]));
    return run_maybe_graph(c, key, enqueue);
}

namespace {

// the orientation table of p slices in the context's buffer
int orient_table(cpra_b200_ctx* c, const void* angles, const void* rot, uint64_t p) {
    int r = ensure_buffer(c, &c->otab, &c->otab_bytes, orient_table_bytes(c->dbl, p), "cudaMalloc(orientation table)");
    if (r) return r;
    CPRA_CHECK_CUDA(launch_orient_table(c->dbl, angles, rot, c->otab, p, c->stream), "orientation table");
    return CPRA_B200_OK;
}

// buffers of the loss and its gradients: G (work), the reductions (three
// sums per slice), the direction table; returns it (null above its limit)
int loss_buffers(cpra_b200_ctx* c, uint64_t m, uint64_t n, uint64_t p, void** atab) {
    int r = ensure_work(c, p * n * m * c->csize());
    if (r) return r;
    r = ensure_reduction(c, 2 * p);  // 2 * CONVERGE_BLOCKS * 2p >= 3 partials per block and slice
    if (r) return r;
    *atab = nullptr;
    if (p <= (uint64_t)ANGLE_TABLE_MAX) {
        r = ensure_buffer(c, &c->atab, &c->atab_bytes, angle_table_bytes(p), "cudaMalloc(angle table)");
        if (r) return r;
        *atab = c->atab;
    }
    return CPRA_B200_OK;
}

// the per-slice sums of the last loss evaluation to the host
int loss_to_host(cpra_b200_ctx* c, uint64_t p, double* loss_host, double* ga_host, double* gr_host) {
    CPRA_CHECK_CUDA(cudaMemcpyAsync(c->host_sums, c->sums, sizeof(double) * 3 * p, cudaMemcpyDeviceToHost, c->stream),
                    "slice_loss_grad");
    CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "slice_loss_grad");
    double loss = 0.0;
    for (uint64_t i = 0; i < p; ++i) {
        loss += c->host_sums[3 * i];
        if (ga_host) ga_host[i] = c->host_sums[3 * i + 1];
        if (gr_host) gr_host[i] = c->host_sums[3 * i + 2];
    }
    if (loss_host) *loss_host = loss;
    return CPRA_B200_OK;
}

bool volume_fft_ok(cpra_b200_ctx* c, uint64_t m, uint64_t n, uint64_t l) {
    auto p2 = [](uint64_t v) { return v >= 2 && (v & (v - 1)) == 0 && v <= 1024; };
    return c->m == m && c->n == n && c->l == l && p2(m) && p2(n) && p2(l);
}

// Forward3D of one real volume into the complex buffer VF
int volume_forward(cpra_b200_ctx* c, const void* vol, void* VF, uint64_t vox) {
    CPRA_CHECK_CUDA(launch_real_complex(c->dbl, true, const_cast<void*>(vol), VF, 1.0, vox, c->stream), "volume");
    CPRA_CHECK_CUDA(launch_fft3d(c->dbl, VF, c->m, c->n, c->l, 1, false, 1.0, twiddles(c, c->m), twiddles(c, c->n),
                                 twiddles(c, c->l), c->work, c->stream),
                    "volume Forward3D");
    return CPRA_B200_OK;
}

// grad_vol = Re(Forward3D^H gV): the adjoint of the shifted unnormalised
// transform is the inverse transform without its 1/(m n l)
int volume_adjoint(cpra_b200_ctx* c, void* gV, void* grad_vol, uint64_t vox) {
    CPRA_CHECK_CUDA(launch_fft3d(c->dbl, gV, c->m, c->n, c->l, 1, true, 1.0, twiddles(c, c->m), twiddles(c, c->n),
                                 twiddles(c, c->l), c->work, c->stream),
                    "volume adjoint");
    CPRA_CHECK_CUDA(launch_real_complex(c->dbl, false, grad_vol, gV, 1.0, vox, c->stream), "volume adjoint");
    return CPRA_B200_OK;
}

}  // namespace

int cpra_b200_slice_orient(cpra_b200_ctx* c, const void* V, const void* angles, const void* rot, uint64_t m, uint64_t n,
                           uint64_t p, uint64_t l, void* slices) {
    CTX_OR_RETURN(c);
    if (!V || !angles || !slices) return fail(CPRA_B200_EARG, "slice: null pointer");
    if (m == 0 || n == 0 || p == 0 || l == 0) return fail(CPRA_B200_EARG, "slice: zero size");
    int r = flush(c);
    if (r) return take_deferred(c);
    r = orient_table(c, angles, rot, p);
    if (r) return r;
    CPRA_CHECK_CUDA(launch_slice(c->dbl, V, c->otab, slices, m, n, p, l, c->stream), "slice");
    return CPRA_B200_OK;
}

int cpra_b200_slice(cpra_b200_ctx* c, const void* V, const void* angles, uint64_t m, uint64_t n, uint64_t p,
                    uint64_t l, void* slices) {
    return cpra_b200_slice_orient(c, V, angles, nullptr, m, n, p, l, slices);
}

int cpra_b200_slice_loss_grad_orient(cpra_b200_ctx* c, const void* V, const void* angles, const void* rot,
                                     const void* A, uint64_t m, uint64_t n, uint64_t p, uint64_t l, void* grad_V,
                                     double* loss_host, double* grad_angles_host, double* grad_rot_host) {
    CTX_OR_RETURN(c);
    if (!V || !angles || !A || !grad_V) return fail(CPRA_B200_EARG, "slice_loss_grad: null pointer");
    if (m == 0 || n == 0 || p == 0 || l == 0) return fail(CPRA_B200_EARG, "slice_loss_grad: zero size");
    if (p > 65535) return fail(CPRA_B200_EUNSUP, "slice_loss_grad: more than 65535 slices");
    int r = flush(c);
    if (r) return take_deferred(c);
    void* atab = nullptr;
    r = loss_buffers(c, m, n, p, &atab);
    if (r) return r;
    r = orient_table(c, angles, rot, p);
    if (r) return r;
    CPRA_CHECK_CUDA(launch_slice_loss_grad(c->dbl, V, angles, c->otab, A, c->work, grad_V, m, n, p, l, c->partials,
                                           c->sums, atab, c->stream),
                    "slice_loss_grad");
    return loss_to_host(c, p, loss_host, grad_angles_host, grad_rot_host);
}

int cpra_b200_slice_loss_grad(cpra_b200_ctx* c, const void* V, const void* angles, const void* A, uint64_t m,
                              uint64_t n, uint64_t p, uint64_t l, void* grad_V, double* loss_host,
                              double* grad_angles_host) {
    return cpra_b200_slice_loss_grad_orient(c, V, angles, nullptr, A, m, n, p, l, grad_V, loss_host, grad_angles_host,
                                            nullptr);
}

int cpra_b200_volume_loss_grad(cpra_b200_ctx* c, const void* vol, const void* angles, const void* rot, const void* A,
                               uint64_t m, uint64_t n, uint64_t p, uint64_t l, void* grad_vol, double* loss_host,
                               double* grad_angles_host, double* grad_rot_host) {
    CTX_OR_RETURN(c);
    if (!vol || !angles || !A || !grad_vol) return fail(CPRA_B200_EARG, "volume_loss_grad: null pointer");
    if (m == 0 || n == 0 || p == 0 || l == 0) return fail(CPRA_B200_EARG, "volume_loss_grad: zero size");
    if (p > 65535) return fail(CPRA_B200_EUNSUP, "volume_loss_grad: more than 65535 slices");
    if (!volume_fft_ok(c, m, n, l))
        return fail(CPRA_B200_EUNSUP, "volume_loss_grad: the context's (m, n, l) must be the volume's, powers of two "
                                      "2..1024");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t vox = l * n * m;
    r = ensure_buffer(c, &c->refine_buf, &c->refine_bytes, 2 * vox * c->csize(), "cudaMalloc(volume buffers)");
    if (r) return r;
    void* atab = nullptr;
    r = loss_buffers(c, m, n, p, &atab);
    if (r) return r;
    r = orient_table(c, angles, rot, p);
    if (r) return r;
    char* buf = static_cast<char*>(c->refine_buf);
    void* VF = buf;
    void* gV = buf + vox * c->csize();
    r = volume_forward(c, vol, VF, vox);
    if (r) return r;
    CPRA_CHECK_CUDA(launch_slice_loss_grad(c->dbl, VF, angles, c->otab, A, c->work, gV, m, n, p, l, c->partials,
                                           c->sums, atab, c->stream),
                    "volume_loss_grad");
    r = volume_adjoint(c, gV, grad_vol, vox);
    if (r) return r;
    return loss_to_host(c, p, loss_host, grad_angles_host, grad_rot_host);
}

int cpra_b200_refine_orient(cpra_b200_ctx* c, void* V, int real_space, void* angles, void* rot, const void* A,
                            uint64_t m, uint64_t n, uint64_t p, uint64_t l, int steps, double lr_volume,
                            double lr_angle, double lr_rot, double* loss_host) {
    CTX_OR_RETURN(c);
    if (!V || !angles || !A) return fail(CPRA_B200_EARG, "refine: null pointer");
    if (m == 0 || n == 0 || p == 0 || l == 0 || steps < 0) return fail(CPRA_B200_EARG, "refine: zero size or steps < 0");
    if (p > 65535) return fail(CPRA_B200_EUNSUP, "refine: more than 65535 slices");
    if (real_space && !volume_fft_ok(c, m, n, l))
        return fail(CPRA_B200_EUNSUP, "refine: a real-space volume needs the context's (m, n, l) to be the volume's, "
                                      "powers of two 2..1024");
    int r = flush(c);
    if (r) return take_deferred(c);
    if (steps == 0) return CPRA_B200_OK;
    const uint64_t vox = l * n * m;
    const uint64_t nv = real_space ? vox : 2 * vox;  // reals refined
    // gV (complex), VF (complex, real-space only), the real gradient
    // (real-space only), the Adam moments, the per-step losses
    const uint64_t cb = (vox * c->csize() + 255) / 256 * 256;
    const uint64_t rb = real_space ? (vox * c->esize() + 255) / 256 * 256 : 0;
    const uint64_t mbytes = (2 * nv + 4 * p) * c->esize();
    const uint64_t gofs = 0, fofs = cb, rofs = fofs + (real_space ? cb : 0), mofs = rofs + rb;
    const uint64_t lofs = mofs + (mbytes + 255) / 256 * 256;
    r = ensure_buffer(c, &c->refine_buf, &c->refine_bytes, lofs + sizeof(double) * (uint64_t)steps,
                      "cudaMalloc(refine buffers)");
    if (r) return r;
    void* atab = nullptr;
    r = loss_buffers(c, m, n, p, &atab);
    if (r) return r;
    char* buf = static_cast<char*>(c->refine_buf);
    void* gV = buf + gofs;
    void* VF = real_space ? buf + fofs : V;
    void* greal = real_space ? buf + rofs : nullptr;
    void* mom = buf + mofs;
    double* loss_dev = reinterpret_cast<double*>(buf + lofs);
    CPRA_CHECK_CUDA(cudaMemsetAsync(mom, 0, mbytes, c->stream), "refine");
    for (int k = 1; k <= steps; ++k) {
        // the iterates are recomputed each step: orientation table, Fourier
        // volume, slices and residuals
        r = orient_table(c, angles, rot, p);
        if (r) return r;
        if (real_space) {
            r = volume_forward(c, V, VF, vox);
            if (r) return r;
        }
        CPRA_CHECK_CUDA(launch_slice_loss_grad(c->dbl, VF, angles, c->otab, A, c->work, gV, m, n, p, l, c->partials,
                                               c->sums, atab, c->stream),
                        "refine");
        if (real_space) {
            r = volume_adjoint(c, gV, greal, vox);
            if (r) return r;
        }
        CPRA_CHECK_CUDA(launch_refine_step(c->dbl, V, nv, angles, rot, real_space ? greal : gV, mom, p, c->sums,
                                           lr_volume, lr_angle, lr_rot, k, loss_dev + (k - 1), c->stream),
                        "refine");
    }
    if (loss_host) {
        CPRA_CHECK_CUDA(cudaMemcpyAsync(loss_host, loss_dev, sizeof(double) * steps, cudaMemcpyDeviceToHost, c->stream),
                        "refine");
        CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "refine");
    }
    return CPRA_B200_OK;
}

int cpra_b200_refine(cpra_b200_ctx* c, void* V, void* angles, const void* A, uint64_t m, uint64_t n, uint64_t p,
                     uint64_t l, int steps, double lr_volume, double lr_angle, double* loss_host) {
    return cpra_b200_refine_orient(c, V, 0, angles, nullptr, A, m, n, p, l, steps, lr_volume, lr_angle, 0.0,
                                   loss_host);
}

int cpra_b200_best_start(cpra_b200_ctx* c, const void* x, const void* A, uint64_t P, uint64_t batch,
                         double* scores_host, uint64_t* best_host, void* best_out) {
    CTX_OR_RETURN(c);
    if (!x || !A || !best_host) return fail(CPRA_B200_EARG, "best_start: null pointer");
    if (P == 0 || batch == 0) return fail(CPRA_B200_EARG, "best_start: P and batch must be positive");
    if (batch > 65535) return fail(CPRA_B200_EUNSUP, "best_start: batch above 65535");
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n))
        return fail(CPRA_B200_EUNSUP, "best_start: each plane size must be 1 or even and at most 4096");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t plane = c->plane(), bytes = batch * plane * c->csize();
    r = ensure_reduction(c, batch);
    if (r) return r;
    r = ensure_work(c, 2 * bytes);
    if (r) return r;
    r = ensure_buffer(c, &c->best_sums, &c->best_bytes, sizeof(double) * 2 * P * batch, "cudaMalloc(best_start sums)");
    if (r) return r;
    char* F = static_cast<char*>(c->work);
    double* sums = static_cast<double*>(c->best_sums);
    for (uint64_t p = 0; p < P; ++p) {
        CPRA_CHECK_CUDA(cudaMemcpyAsync(F, static_cast<const char*>(x) + p * bytes, bytes, cudaMemcpyDefault, c->stream),
                        "best_start");
        CPRA_CHECK_CUDA(launch_fft2d(c->dbl, F, c->m, c->n, batch, false, 1.0, twiddles(c, c->m), twiddles(c, c->n),
                                     F + bytes, c->stream),
                        "best_start");
        CPRA_CHECK_CUDA(launch_rfactor_sums(c->dbl, F, static_cast<const char*>(A) + p * plane * c->esize(), 0, plane,
                                            batch, c->partials, sums + 2 * batch * p, c->stream),
                        "best_start");
    }
    std::vector<double> h(2 * P * batch);
    CPRA_CHECK_CUDA(cudaMemcpyAsync(h.data(), sums, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream),
                    "best_start");
    CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "best_start");
    uint64_t best = 0;
    double best_score = 0.0;
    for (uint64_t b = 0; b < batch; ++b) {
        double acc = 0.0;
        for (uint64_t p = 0; p < P; ++p) acc += h[2 * (batch * p + b)] / h[2 * (batch * p + b) + 1];
        const double score = acc / (double)P;
        if (scores_host) scores_host[b] = score;
        if (b == 0 || score < best_score) {
            best = b;
            best_score = score;
        }
    }
    *best_host = best;
    if (best_out) {
        const uint64_t pb = plane * c->csize();
        for (uint64_t p = 0; p < P; ++p)
            CPRA_CHECK_CUDA(cudaMemcpyAsync(static_cast<char*>(best_out) + p * pb,
                                            static_cast<const char*>(x) + (p * batch + best) * pb, pb, cudaMemcpyDefault,
                                            c->stream),
                            "best_start");
    }
    return CPRA_B200_OK;
}

int cpra_b200_kernel_timing(cpra_b200_ctx* c, double* ms, uint64_t* launches, uint64_t* pattern_iters) {
    CTX_OR_RETURN(c);
    int r = flush(c);
    if (r) return take_deferred(c);
    CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "kernel_timing");
    double total = 0.0;
    for (auto& pr : c->timed) {
        float t = 0.0f;
        CPRA_CHECK_CUDA(cudaEventElapsedTime(&t, pr.first, pr.second), "cudaEventElapsedTime");
        total += t;
        c->free_events.push_back(pr.first);
        c->free_events.push_back(pr.second);
    }
    if (ms) *ms = total;
    if (launches) *launches = c->timed.size();
    if (pattern_iters) *pattern_iters = c->timed_pattern_iters;
    c->timed.clear();
    c->timed_pattern_iters = 0;
    return CPRA_B200_OK;
}

// Lanes of cpra_run's wavefront schedule: with CPRA_B200_OPT_LANES 0, as many
// as it takes for the angles running side by side to fill the GPU's resident
// CTA slots one and a half times (one lane when one angle's launch of the
// one-CTA-per-pattern kernel already fills them once: then more lanes only
// compete for L2).  The line passes (256², 512²) take at least four: each
// iteration is a column pass and a row pass that waits for all of it, and the
// episodes beside them fill every pass boundary's drain and ramp (measured by
// the autotuner: 4 lanes ahead of the slot count at 256² and 512², 16 starts).
int run_lanes_for(cpra_b200_ctx* c, uint64_t batch) {
    if (c->lanes_opt > 0) return c->lanes_opt;
    if (!c->fusion || !dm_fusable(c)) return 1;
    uint64_t ctas, per_sm;
    const bool line_passes = !dm_fused_supported(c->dbl, c->m, c->n);
    if (!line_passes) {
        ctas = batch;
        per_sm = (uint64_t)dm_fused_ctas_per_sm(c->m);
    } else {
        ctas = dm_large_row_ctas(c->m, batch);
        per_sm = (uint64_t)dm_large_ctas_per_sm(c->m);
    }
    const uint64_t slots = per_sm * (uint64_t)sm_count();
    uint64_t w = 1;
    if (ctas > 0 && ctas < slots)
        w = std::min<uint64_t>(CPRA_B200_MAX_LANES, (3 * slots + 2 * ctas - 1) / (2 * ctas));
    if (line_passes) w = std::max<uint64_t>(w, 4);
    return (int)w;
}

// Lanes for `epi` episodes: at most `want`, and no more than it takes to give
// each lane the same number of episodes as the busiest one has (a lane takes
// its episodes one after another, so the busiest lane sets the time).
int balanced_lanes(int want, int epi) {
    if (epi <= 1 || want <= 1) return 1;
    const int w = std::min(want, epi);
    const int per_lane = (epi + w - 1) / w;
    return std::max(1, (epi + per_lane - 1) / per_lane);
}

int cpra_b200_get_option(cpra_b200_ctx* c, int option, int64_t* value) {
    CTX_OR_RETURN(c);
    if (!value) return fail(CPRA_B200_EARG, "get_option: null value");
    switch (option) {
        case CPRA_B200_OPT_FUSION: *value = c->fusion ? 1 : 0; break;
        case CPRA_B200_OPT_SPACE_MODE: *value = c->space_mode; break;
        case CPRA_B200_OPT_DATA_MODE: *value = c->data_mode; break;
        case CPRA_B200_OPT_SEED: *value = (int64_t)c->seed; break;
        case CPRA_B200_OPT_KERNEL_TIMING: *value = c->timing ? 1 : 0; break;
        case CPRA_B200_OPT_HIO_CHUNK: *value = (int64_t)c->hio_chunk; break;
        case CPRA_B200_OPT_GRAPH: *value = c->graphs ? 1 : 0; break;
        case CPRA_B200_OPT_LANES:
            *value = (c->autotune && c->lanes_opt == 0 && c->tuned_lanes > 0) ? c->tuned_lanes
                                                                              : run_lanes_for(c, c->batch);
            break;
        case CPRA_B200_OPT_IO_CHUNK: *value = (int64_t)c->io_chunk; break;
        case CPRA_B200_OPT_AUTOTUNE: *value = c->autotune ? 1 : 0; break;
        case CPRA_B200_OPT_TMEM: *value = c->tmem ? 1 : 0; break;
        case CPRA_B200_OPT_FUSED3D: *value = c->fused3d ? 1 : 0; break;
        case CPRA_B200_OPT_HIO_CLUSTER: *value = c->hio_cluster; break;
        case CPRA_B200_OPT_FAILURE_TEST: *value = c->failure_test ? 1 : 0; break;
        default: return fail(CPRA_B200_EARG, "unknown option");
    }
    return CPRA_B200_OK;
}

// lanes 1..W-1 with their streams, scratch and per-angle events (lane 0 is the
// context's own stream and buffers)
int ensure_lanes(cpra_b200_ctx* c, int W, uint64_t drv_bytes, uint64_t work_bytes, uint64_t P) {
    if (W <= 1) return CPRA_B200_OK;
    if (c->run_lanes.size() < (size_t)W) c->run_lanes.resize(W);
    if (!c->lane_fork)
        CPRA_CHECK_CUDA(cudaEventCreateWithFlags(&c->lane_fork, cudaEventDisableTiming), "cudaEventCreate");
    for (int k = 0; k < W; ++k) {
        RunLane& lane = c->run_lanes[k];
        if (k > 0) {
            if (!lane.stream)
                CPRA_CHECK_CUDA(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking), "cudaStreamCreate");
            if (!lane.join)
                CPRA_CHECK_CUDA(cudaEventCreateWithFlags(&lane.join, cudaEventDisableTiming), "cudaEventCreate");
            int r = ensure_buffer(c, &lane.drv, &lane.drv_bytes, drv_bytes, "cudaMalloc(lane buffers)");
            if (!r) r = ensure_buffer(c, &lane.work, &lane.work_bytes, work_bytes, "cudaMalloc(lane work)");
            if (r) return r;
        }
        while (lane.ev.size() < P) {
            cudaEvent_t e;
            CPRA_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
            lane.ev.push_back(e);
        }
    }
    return CPRA_B200_OK;
}

static int cpra_run_impl(cpra_b200_ctx* c, void* x, const void* A, const void* S, uint64_t P, uint64_t batch, int epi,
                         int iters, int pre_iter, double beta, int final_step, void* err_host,
                         const cudaEvent_t* ready, const cudaEvent_t* done,
                         const std::function<int()>& after_enqueue = {});

// CPRA_B200_OPT_AUTOTUNE: the lane count of cpra_run's wavefront schedule,
// measured.  Every candidate (1 to 4 lanes and the automatic choice, as many
// as the episodes allow after balancing) runs the same min(epi, 4) episodes
// on a copy of x, timed by CUDA events on the context's stream, graphs off;
// the largest candidate runs first and again at the end, so that its first
// run carries the lanes' one-time set-up.  Lane counts change the schedule
// only, never the results, so the choice is free.
static int tune_lanes(cpra_b200_ctx* c, const void* x, const void* A, const void* S, uint64_t P, uint64_t batch,
                      int epi, int iters, double beta, int* best_out) {
    const uint64_t xbytes = P * batch * c->plane() * c->csize();
    const int E = std::min(epi, 4);
    std::vector<int> cand;
    for (int w : {1, 2, 3, 4, run_lanes_for(c, batch)}) {
        const int eff = balanced_lanes(std::min(w, CPRA_B200_MAX_LANES), E);
        if (std::find(cand.begin(), cand.end(), eff) == cand.end()) cand.push_back(eff);
    }
    std::sort(cand.rbegin(), cand.rend());
    if (cand.size() == 1) {
        *best_out = cand[0];
        return CPRA_B200_OK;
    }
    struct Restore {
        cpra_b200_ctx* c;
        int lanes;
        bool graphs, timing;
        void* trial = nullptr;
        cudaEvent_t ev[2] = {nullptr, nullptr};
        ~Restore() {
            c->lanes_opt = lanes;
            c->graphs = graphs;
            c->timing = timing;
            if (trial) {
                cudaStreamSynchronize(c->stream);
                cudaFree(trial);
            }
            for (cudaEvent_t e : ev)
                if (e) cudaEventDestroy(e);
        }
    } g{c, c->lanes_opt, c->graphs, c->timing};
    c->graphs = false;
    c->timing = false;
    if (cudaMalloc(&g.trial, xbytes) != cudaSuccess) {
        // no room for the copy: keep the heuristic's choice for this key (an
        // out-of-memory error is not sticky; clear it)
        cudaGetLastError();
        g.trial = nullptr;
        *best_out = run_lanes_for(c, batch);
        return CPRA_B200_OK;
    }
    CPRA_CHECK_CUDA(cudaEventCreate(&g.ev[0]), "cudaEventCreate");
    CPRA_CHECK_CUDA(cudaEventCreate(&g.ev[1]), "cudaEventCreate");
    std::vector<float> ms(cand.size(), 0.0f);
    for (size_t i = 0; i <= cand.size(); ++i) {
        const size_t k = (i == cand.size()) ? 0 : i;
        c->lanes_opt = cand[k];
        CPRA_CHECK_CUDA(cudaMemcpyAsync(g.trial, x, xbytes, cudaMemcpyDeviceToDevice, c->stream), "autotune");
        CPRA_CHECK_CUDA(cudaEventRecord(g.ev[0], c->stream), "autotune");
        int r = cpra_run_impl(c, g.trial, A, S, P, batch, E, iters, 0, beta, 0, nullptr, nullptr, nullptr);
        if (r) return r;
        CPRA_CHECK_CUDA(cudaEventRecord(g.ev[1], c->stream), "autotune");
        CPRA_CHECK_CUDA(cudaEventSynchronize(g.ev[1]), "autotune");
        CPRA_CHECK_CUDA(cudaEventElapsedTime(&ms[k], g.ev[0], g.ev[1]), "autotune");
    }
    size_t best = 0;
    for (size_t k = 1; k < cand.size(); ++k)
        if (ms[k] < ms[best]) best = k;
    *best_out = cand[best];
    return CPRA_B200_OK;
}

// The carousel driver on device buffers.  ready (optional, P events): angle
// p's plane of x is complete once ready[p] has fired; the first episode (and
// the pre-iterations) wait for each plane they read, just before its first
// use.  done (optional, P events): recorded after angle p's final projection.
// after_enqueue (optional) runs once all the work is enqueued, before the
// wait for the error sums.
static int cpra_run_impl(cpra_b200_ctx* c, void* x, const void* A, const void* S, uint64_t P, uint64_t batch, int epi,
                         int iters, int pre_iter, double beta, int final_step, void* err_host,
                         const cudaEvent_t* ready, const cudaEvent_t* done,
                         const std::function<int()>& after_enqueue) {
    if (!x || !A || !S) return fail(CPRA_B200_EARG, "cpra_run: null pointer");
    if (P < 2) return fail(CPRA_B200_EARG, "cpra_run: P >= 2 (the carousel mix reads angles p-1 and p+1)");
    if (batch != c->batch) return fail(CPRA_B200_EARG, "cpra_run: batch must equal the context's batch_size");
    if (epi < 0 || iters < 0 || pre_iter < 0) return fail(CPRA_B200_EARG, "cpra_run: negative count");
    if (err_host && epi > 0 && iters < 1) return fail(CPRA_B200_EARG, "cpra_run: the error step needs iters >= 1");
    const double b = c->round_t(beta);
    if (b == 0.0) return fail(CPRA_B200_EARG, "cpra_run: beta == 0");
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n))
        return fail(CPRA_B200_EUNSUP, "cpra_run: each plane size must be 1 or even and at most 4096");
    int r = flush(c);
    if (r) return take_deferred(c);
    // CPRA_B200_OPT_AUTOTUNE: the measured lane count of this run's key.  A
    // host-buffer run (x still arriving) uses the cache but does not tune.
    int tuned = 0;
    if (c->autotune && c->lanes_opt == 0 && epi > 1 && !c->capturing) {
        const std::string key = graph_key("lanes", c->m, c->n, batch, P, iters, c->fusion, c->space_mode,
                                          c->data_mode, c->dbl);
        for (const auto& e : c->tune_cache)
            if (e.first == key) tuned = e.second;
        if (!tuned && !ready) {
            if ((r = tune_lanes(c, x, A, S, P, batch, epi, iters, beta, &tuned))) return r;
            c->tune_cache.emplace_back(key, tuned);
        }
        c->tuned_lanes = tuned;
    }
    const uint64_t MN = c->plane(), MNB = MN * batch;
    const uint64_t cb = MNB * c->csize();
    if ((r = ensure_buffer(c, &c->drv, &c->drv_bytes, 3 * cb, "cudaMalloc(driver buffers)"))) return r;
    const bool want_err = err_host && epi > 0;
    if (want_err) {
        r = ensure_reduction(c, batch);
        if (r) return r;
        if (c->err_cap < P * batch) {
            ++c->epoch;
            if (c->err_sums) {
                cudaStreamSynchronize(c->stream);
                cudaFree(c->err_sums);
                cudaFreeHost(c->host_err);
                c->err_sums = c->host_err = nullptr;
                c->err_cap = 0;
            }
            CPRA_CHECK_CUDA(cudaMalloc(&c->err_sums, sizeof(double) * 2 * P * batch), "cudaMalloc(errors)");
            CPRA_CHECK_CUDA(cudaMallocHost(&c->host_err, sizeof(double) * 2 * P * batch), "cudaMallocHost(errors)");
            c->err_cap = P * batch;
        }
    }
    // scratch of the fused large-plane iterations and of non-power-of-two
    // transforms, reserved before any work is enqueued (and before a capture)
    uint64_t work_need = batch * MN * c->csize();
    if (dm_fusable(c) && !dm_fused_supported(c->dbl, c->m, c->n))
        work_need = std::max(work_need, dm_large_scratch_bytes(c->m, c->n, batch, 0));
    r = ensure_work(c, work_need);
    if (r) return r;
    // lanes of the wavefront schedule, each with its own scratch
    const int W = balanced_lanes(tuned ? tuned : run_lanes_for(c, batch), epi);
    if ((r = ensure_lanes(c, W, 3 * cb, work_need, P))) return r;
    char* base = static_cast<char*>(x);
    const char* Ab = static_cast<const char*>(A);
    const char* Sb = static_cast<const char*>(S);
    const uint64_t rb = MN * c->esize();
    auto xp = [&](uint64_t p) { return static_cast<void*>(base + cb * p); };
    // src/CPRA_MKL.cpp:98,103,109,110: coefficients in double from a T beta, passed as T
    const DmCoef coef = {c->round_t(-1.0 / b), c->round_t(1.0 + 1.0 / b), c->round_t(1.0 / b), c->round_t(1.0 - 1.0 / b),
                         c->round_t(b),        1.0,                         c->round_t(-1.0 * b), 1.0};
    // a lane's t1, t2, old and its scope: lane k > 0 runs on its own stream
    // with its own work buffer (swapped into the context while it is issued)
    struct LaneBufs {
        char *t1, *t2, *old;
    };
    auto bufs = [&](int k) {
        char* d = static_cast<char*>(k == 0 ? c->drv : c->run_lanes[k].drv);
        return LaneBufs{d, d + cb, d + 2 * cb};
    };
    struct LaneScope {
        cpra_b200_ctx* c;
        RunLane* lane;
        cudaStream_t stream;
        void* work;
        uint64_t work_bytes;
        LaneScope(cpra_b200_ctx* c_, int k) : c(c_), lane(k ? &c_->run_lanes[k] : nullptr) {
            stream = c->stream;
            work = c->work;
            work_bytes = c->work_bytes;
            if (lane) {
                c->stream = lane->stream;
                c->work = lane->work;
                c->work_bytes = lane->work_bytes;
            }
        }
        ~LaneScope() {
            if (lane) {
                lane->work = c->work;
                lane->work_bytes = c->work_bytes;
                c->stream = stream;
                c->work = work;
                c->work_bytes = work_bytes;
            }
        }
    };
    char* t1 = bufs(0).t1;
    char* t2 = bufs(0).t2;
    auto pattern = [&](uint64_t p, uint64_t cp, const LaneBufs& lb) {
        DmPattern d;
        d.x = xp(p);
        d.t1 = lb.t1;
        d.t2 = lb.t2;
        d.A = Ab + rb * cp;
        d.S = Sb + rb * cp;
        d.num = MNB;
        d.batch = batch;
        d.c = coef;
        return d;
    };
    auto copy = [&](void* dst, const void* src) {
        return cudaMemcpyAsync(dst, src, cb, cudaMemcpyDeviceToDevice, c->stream);
    };
    auto enqueue = [&]() -> int {
    int r = CPRA_B200_OK;
    auto await = [&](uint64_t p) -> int {
        if (ready) CPRA_CHECK_CUDA(cudaStreamWaitEvent(c->stream, ready[p < P ? p : P - 1], 0), "cpra_run");
        return CPRA_B200_OK;
    };
    if (ready) {
        // Step A reads angle 0; angle 0 of the first episode also reads angle 1
        if ((r = await(0))) return r;
    }
    // Step A (:35-55): pre-reconstruction of angle 0 with the first constraint planes
    if (pre_iter > 0) {
        CPRA_CHECK_CUDA(copy(t1, xp(0)), "cpra_run");
        CPRA_CHECK_CUDA(copy(t2, xp(0)), "cpra_run");
        if ((r = dm_any(c, pattern(0, 0, bufs(0)), pre_iter))) return r;
    }
    // one angle of an episode (src/CPRA_MKL.cpp:63-123)
    auto run_angle = [&](int e, uint64_t p, const LaneBufs& lb) -> int {
        int r = CPRA_B200_OK;
        char* t1 = lb.t1;
        char* t2 = lb.t2;
        char* old = lb.old;
        const DmPattern pat = pattern(p, p, lb);
        const bool err_here = want_err && e == epi - 1;
        const bool fused = iters > 0 && dm_fusable(c);
        if (fused && (!err_here || iters >= 2)) {
            // carousel mix, t1 = t2 = x and the angle's iterations (all but
            // the last one on an error-reporting angle) in one launch
            const int mix = (p == 0) ? MIX_FIRST : (p == P - 1) ? MIX_LAST : MIX_MIDDLE;
            if ((r = launch_fused(c, pat, err_here ? iters - 1 : iters, mix, p > 0 ? xp(p - 1) : nullptr,
                                  p + 1 < P ? xp(p + 1) : nullptr, 1)))
                return r;
            if (!err_here) return CPRA_B200_OK;
        } else {
            if (p == P - 1) {
                CPRA_CHECK_CUDA(launch_merge_add(c->dbl, xp(p - 1), xp(p), 0.5, 0.5, MNB, c->stream), "cpra_run");
            } else if (p == 0) {
                CPRA_CHECK_CUDA(launch_merge_add(c->dbl, xp(p + 1), xp(p), 0.5, 0.5, MNB, c->stream), "cpra_run");
            } else {
                CPRA_CHECK_CUDA(launch_merge_add(c->dbl, xp(p - 1), xp(p), 0.5, 0.0, MNB, c->stream), "cpra_run");
                CPRA_CHECK_CUDA(launch_merge_add(c->dbl, xp(p + 1), xp(p), 0.5, 1.0, MNB, c->stream), "cpra_run");
            }
            CPRA_CHECK_CUDA(copy(t1, xp(p)), "cpra_run");
            CPRA_CHECK_CUDA(copy(t2, xp(p)), "cpra_run");
            if (!err_here) {
                if ((r = dm_any(c, pat, iters))) return r;
                return CPRA_B200_OK;
            }
            if ((r = dm_any(c, pat, iters - 1))) return r;
        }
        CPRA_CHECK_CUDA(copy(old, xp(p)), "cpra_run");
        if ((r = dm_any(c, pat, 1))) return r;
        CPRA_CHECK_CUDA(copy(t1, xp(p)), "cpra_run");
        if ((r = run_fft2d(c, old, false))) return r;
        if ((r = run_fft2d(c, t1, false))) return r;
        // ConvergeError (CUDA_Impl.inl:145-172): old <- t1 - old, ||old_i|| / ||t1_i||
        CPRA_CHECK_CUDA(launch_merge_add(c->dbl, t1, old, 1.0, -1.0, MNB, c->stream), "cpra_run");
        CPRA_CHECK_CUDA(launch_norm_pairs(c->dbl, old, t1, MN, MN, batch, c->partials, c->err_sums + 2 * batch * p,
                                          c->stream),
                        "cpra_run");
        return CPRA_B200_OK;
    };
    // final projection of one angle (:126-140)
    auto final_projection = [&](uint64_t p, const LaneBufs& lb) -> int {
        int r = CPRA_B200_OK;
        char* t1 = lb.t1;
        const DmPattern pat = pattern(p, p, lb);
        CPRA_CHECK_CUDA(copy(t1, xp(p)), "cpra_run");
        const Op seq[5] = {{OpKind::Fwd2D, t1, nullptr, 0, 0, 0, 0},
                           {OpKind::DataReal, t1, pat.A, MNB, batch, 0, 0},
                           {OpKind::Bwd2D, t1, nullptr, 0, 0, 0, 0},
                           {OpKind::Merge, t1, xp(p), MNB, 1, coef.a1, coef.b1},
                           {OpKind::Space, t1, pat.S, MNB, batch, 0, 0}};
        for (const Op& op : seq)
            if ((r = exec_op(c, op))) return r;
        CPRA_CHECK_CUDA(copy(xp(p), t1), "cpra_run");
        if (done) CPRA_CHECK_CUDA(cudaEventRecord(done[p], c->stream), "cpra_run");
        return CPRA_B200_OK;
    };
    // Step B (:59-124).  The final projection of angle p depends on x[p] alone
    // and nothing of the last episode reads x[p] after angle p + 1 has run, so
    // it is issued right there: the same operations on the same data as after
    // the loop (:126-140), with each angle's result complete early.
    //
    // Angle p of episode e reads x[p-1], x[p], x[p+1] and writes x[p]: it
    // needs angle p-1 of episode e and angle p+1 of episode e-1 done, and
    // nothing else (every other order constraint follows from those two).
    // With W > 1 lanes, episode e runs on lane e mod W and the angles are
    // issued in wavefront order (p + 2e ascending), so angle p of episode e
    // runs beside angle p-2 of episode e+1; each angle reads exactly the data
    // it reads in the sequential order, so the results are the same bits.
    auto issue = [&](int e, uint64_t p) -> int {
        const int k = e % W;
        LaneScope scope(c, k);
        int r = CPRA_B200_OK;
        if (e == 0 && (r = await(p + 1))) return r;
        if (W > 1 && e > 0 && p + 1 < P && (e - 1) % W != k)
            CPRA_CHECK_CUDA(cudaStreamWaitEvent(c->stream, c->run_lanes[(e - 1) % W].ev[p + 1], 0), "cpra_run");
        const LaneBufs lb = bufs(k);
        if ((r = run_angle(e, p, lb))) return r;
        if (W > 1 && e + 1 < epi && p > 0 && (e + 1) % W != k)
            CPRA_CHECK_CUDA(cudaEventRecord(c->run_lanes[k].ev[p], c->stream), "cpra_run");
        if (final_step && e == epi - 1) {
            if (p > 0 && (r = final_projection(p - 1, lb))) return r;
            if (p == P - 1 && (r = final_projection(P - 1, lb))) return r;
        }
        return CPRA_B200_OK;
    };
    if (W == 1) {
        for (int e = 0; e < epi; ++e)
            for (uint64_t p = 0; p < P; ++p)
                if ((r = issue(e, p))) return r;
    } else {
        CPRA_CHECK_CUDA(cudaEventRecord(c->lane_fork, c->stream), "cpra_run");
        for (int k = 1; k < W; ++k)
            CPRA_CHECK_CUDA(cudaStreamWaitEvent(c->run_lanes[k].stream, c->lane_fork, 0), "cpra_run");
        const uint64_t steps = P + 2 * (uint64_t)(epi - 1);
        for (uint64_t t = 0; t < steps; ++t)
            for (int e = 0; e < epi; ++e) {
                if (t < 2 * (uint64_t)e) break;
                const uint64_t p = t - 2 * (uint64_t)e;
                if (p < P && (r = issue(e, p))) return r;
            }
        for (int k = 1; k < W; ++k) {
            CPRA_CHECK_CUDA(cudaEventRecord(c->run_lanes[k].join, c->run_lanes[k].stream), "cpra_run");
            CPRA_CHECK_CUDA(cudaStreamWaitEvent(c->stream, c->run_lanes[k].join, 0), "cpra_run");
        }
    }
    if (final_step && epi == 0) {
        if ((r = await(P - 1))) return r;
        for (uint64_t p = 0; p < P; ++p)
            if ((r = final_projection(p, bufs(0)))) return r;
    }
    if (want_err)
        CPRA_CHECK_CUDA(cudaMemcpyAsync(c->host_err, c->err_sums, sizeof(double) * 2 * P * batch,
                                        cudaMemcpyDeviceToHost, c->stream),
                        "cpra_run");
    return CPRA_B200_OK;
    };
    r = (ready || done) ? enqueue()
                        : run_maybe_graph(c,
                                          graph_key("cpra_run", x, A, S, P, batch, epi, iters, pre_iter, b,
                                                    final_step, want_err, c->space_mode, c->data_mode, c->fusion, W,
                                                    c->tmem),
                                          enqueue);
    if (r) return r;
    if (after_enqueue && (r = after_enqueue())) return r;
    if (want_err) {
        CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "cpra_run");
        for (uint64_t i = 0; i < P * batch; ++i) {
            const double v = std::sqrt(c->host_err[2 * i]) / std::sqrt(c->host_err[2 * i + 1]);
            if (c->dbl)
                static_cast<double*>(err_host)[i] = v;
            else
                static_cast<float*>(err_host)[i] = (float)v;
        }
    }
    return CPRA_B200_OK;
}


int cpra_b200_cpra_run(cpra_b200_ctx* c, void* x, const void* A, const void* S, uint64_t P, uint64_t batch, int epi,
                       int iters, int pre_iter, double beta, int final_step, void* err_host) {
    CTX_OR_RETURN(c);
    return cpra_run_impl(c, x, A, S, P, batch, epi, iters, pre_iter, beta, final_step, err_host, nullptr, nullptr);
}

int cpra_b200_cpra_run_host(cpra_b200_ctx* c, void* x_host, const void* A_host, const void* S_host, uint64_t P,
                            uint64_t batch, int epi, int iters, int pre_iter, double beta, int final_step,
                            void* err_host) {
    CTX_OR_RETURN(c);
    if (!x_host || !A_host || !S_host) return fail(CPRA_B200_EARG, "cpra_run_host: null pointer");
    if (P < 2 || batch != c->batch) return fail(CPRA_B200_EARG, "cpra_run_host: P >= 2 and batch == batch_size");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t cb = c->plane() * batch * c->csize(), rb = c->plane() * c->esize();
    if ((r = ensure_buffer(c, &c->hx, &c->hx_bytes, P * cb, "cudaMalloc(cpra_run_host x)"))) return r;
    if ((r = ensure_buffer(c, &c->hA, &c->hA_bytes, P * rb, "cudaMalloc(cpra_run_host A)"))) return r;
    if ((r = ensure_buffer(c, &c->hS, &c->hS_bytes, P * rb, "cudaMalloc(cpra_run_host S)"))) return r;
    if (!c->copy_stream)
        CPRA_CHECK_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    while (c->run_events.size() < 2 * P + 1) {
        cudaEvent_t e;
        CPRA_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        c->run_events.push_back(e);
    }
    const cudaEvent_t* ready = c->run_events.data();
    const cudaEvent_t* done = ready + P;
    const cudaEvent_t start = ready[2 * P];
    char* hx = static_cast<char*>(c->hx);
    char* xh = static_cast<char*>(x_host);
    // uploads on the copy stream once the context's earlier work is done, angle
    // by angle (x, A and S of angle p, then ready[p]); the driver waits for
    // angle p + 1 before it runs angle p of the first episode
    CPRA_CHECK_CUDA(cudaEventRecord(start, c->stream), "cpra_run_host");
    CPRA_CHECK_CUDA(cudaStreamWaitEvent(c->copy_stream, start, 0), "cpra_run_host");
    for (uint64_t p = 0; p < P; ++p) {
        CPRA_CHECK_CUDA(cudaMemcpyAsync(hx + p * cb, xh + p * cb, cb, cudaMemcpyHostToDevice, c->copy_stream),
                        "cpra_run_host");
        CPRA_CHECK_CUDA(cudaMemcpyAsync(static_cast<char*>(c->hA) + p * rb, static_cast<const char*>(A_host) + p * rb,
                                        rb, cudaMemcpyHostToDevice, c->copy_stream),
                        "cpra_run_host");
        CPRA_CHECK_CUDA(cudaMemcpyAsync(static_cast<char*>(c->hS) + p * rb, static_cast<const char*>(S_host) + p * rb,
                                        rb, cudaMemcpyHostToDevice, c->copy_stream),
                        "cpra_run_host");
        CPRA_CHECK_CUDA(cudaEventRecord(ready[p], c->copy_stream), "cpra_run_host");
    }
    // downloads: angle p as soon as its final projection is done (all at the
    // end without the final projection)
    auto download = [&]() -> int {
        for (uint64_t p = 0; p < P; ++p) {
            if (final_step || p == 0) {
                if (!final_step) CPRA_CHECK_CUDA(cudaEventRecord(done[0], c->stream), "cpra_run_host");
                CPRA_CHECK_CUDA(cudaStreamWaitEvent(c->copy_stream, done[final_step ? p : 0], 0), "cpra_run_host");
            }
            CPRA_CHECK_CUDA(cudaMemcpyAsync(xh + p * cb, hx + p * cb, cb, cudaMemcpyDeviceToHost, c->copy_stream),
                            "cpra_run_host");
        }
        return CPRA_B200_OK;
    };
    r = cpra_run_impl(c, c->hx, c->hA, c->hS, P, batch, epi, iters, pre_iter, beta, final_step, err_host, ready,
                      final_step ? done : nullptr, download);
    const cudaError_t e = cudaStreamSynchronize(c->copy_stream);
    if (r) return r;
    CPRA_CHECK_CUDA(e, "cpra_run_host");
    CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "cpra_run_host");
    return CPRA_B200_OK;
}


// The conventional 3D driver ShrinkWrap_CONV_MKL_Sample (src/CONV_MKL.cpp:10-88)
// on device buffers: x holds the context's batch of [l][m][n] volumes, A and S
// one volume each (broadcast over the batch, as the reference's calls do).
//   t1 = t2 = x (:31-32); `iters` difference-map iterations with Forward3D /
//   Backward3D (:35-67; fused into axis passes for power-of-two volumes);
//   on the last one, the convergence error (:39-44, 70-77) when err_host is
//   given; then, with final_step, the final projection (:80-88).
static int conv_run_impl(cpra_b200_ctx* c, void* x, const void* A, const void* S, int iters, double beta,
                         int final_step, void* err_host) {
    if (!x || !A || !S) return fail(CPRA_B200_EARG, "conv_run: null pointer");
    if (iters < 0) return fail(CPRA_B200_EARG, "conv_run: negative count");
    if (err_host && iters < 1) return fail(CPRA_B200_EARG, "conv_run: the error step needs iters >= 1");
    if (err_host && c->batch > 65535) return fail(CPRA_B200_EUNSUP, "conv_run: batch_size above 65535");
    const double b = c->round_t(beta);
    if (b == 0.0) return fail(CPRA_B200_EARG, "conv_run: beta == 0");
    if (!fft_length_supported(c->m) || !fft_length_supported(c->n) || !fft_length_supported(c->l))
        return fail(CPRA_B200_EUNSUP, "conv_run: each size must be 1 or even and at most 4096");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t B = c->batch, MN = c->plane(), vol = MN * c->l, num = vol * B, cb = num * c->csize();
    if ((r = ensure_buffer(c, &c->drv, &c->drv_bytes, 3 * cb, "cudaMalloc(driver buffers)"))) return r;
    const bool want_err = err_host != nullptr;
    if (want_err && (r = ensure_reduction(c, B))) return r;
    if ((r = ensure_work(c, cb))) return r;  // transforms of other sizes
    char* t1 = static_cast<char*>(c->drv);
    char* t2 = t1 + cb;
    char* old = t2 + cb;
    // src/CONV_MKL.cpp:47,53,64,65: the coefficients as the 2D driver's
    const DmCoef coef = {c->round_t(-1.0 / b), c->round_t(1.0 + 1.0 / b), c->round_t(1.0 / b), c->round_t(1.0 - 1.0 / b),
                         c->round_t(b),        1.0,                         c->round_t(-1.0 * b), 1.0};
    DmPattern pat;
    pat.x = x;
    pat.t1 = t1;
    pat.t2 = t2;
    pat.A = A;
    pat.S = S;
    pat.num = num;
    pat.batch = B;
    pat.c = coef;
    pat.dim = 3;
    auto copy = [&](void* dst, const void* src) {
        return cudaMemcpyAsync(dst, src, cb, cudaMemcpyDeviceToDevice, c->stream);
    };
    auto iterate = [&](int n) -> int {
        if (n <= 0) return CPRA_B200_OK;
        if (fusable_shape3d(c)) return launch_fused(c, pat, n);
        for (int i = 0; i < n; ++i) {
            const Op seq[12] = {
                {OpKind::Fwd3D, t1, nullptr, 0, 0, 0, 0},   {OpKind::DataReal, t1, A, num, B, 0, 0},
                {OpKind::Bwd3D, t1, nullptr, 0, 0, 0, 0},   {OpKind::Merge, t1, x, num, 1, coef.a1, coef.b1},
                {OpKind::Space, t1, S, num, B, 0, 0},       {OpKind::Space, t2, S, num, B, 0, 0},
                {OpKind::Merge, t2, x, num, 1, coef.a2, coef.b2}, {OpKind::Fwd3D, t2, nullptr, 0, 0, 0, 0},
                {OpKind::DataReal, t2, A, num, B, 0, 0},    {OpKind::Bwd3D, t2, nullptr, 0, 0, 0, 0},
                {OpKind::Merge, x, t1, num, 1, coef.a3, coef.b3}, {OpKind::Merge, x, t2, num, 1, coef.a4, coef.b4}};
            for (const Op& op : seq) {
                const int rr = exec_op(c, op);
                if (rr) return rr;
            }
        }
        return CPRA_B200_OK;
    };
    auto enqueue = [&]() -> int {
        int r = CPRA_B200_OK;
        CPRA_CHECK_CUDA(copy(t1, x), "conv_run");
        CPRA_CHECK_CUDA(copy(t2, x), "conv_run");
        if ((r = iterate(want_err ? iters - 1 : iters))) return r;
        if (want_err) {
            CPRA_CHECK_CUDA(copy(old, x), "conv_run");
            if ((r = iterate(1))) return r;
            CPRA_CHECK_CUDA(copy(t1, x), "conv_run");
            if ((r = exec_fft3d(c, old, false)) || (r = exec_fft3d(c, t1, false))) return r;
            // ConvergeError (CUDA_Impl.inl:145-172): old <- t1 - old; norms over
            // the first m*n elements of each volume (stride m*n*l)
            CPRA_CHECK_CUDA(launch_merge_add(c->dbl, t1, old, 1.0, -1.0, num, c->stream), "conv_run");
            CPRA_CHECK_CUDA(launch_norm_pairs(c->dbl, old, t1, MN, vol, B, c->partials, c->sums, c->stream),
                            "conv_run");
            CPRA_CHECK_CUDA(cudaMemcpyAsync(c->host_sums, c->sums, sizeof(double) * 2 * B, cudaMemcpyDeviceToHost,
                                            c->stream),
                            "conv_run");
        }
        if (final_step) {
            CPRA_CHECK_CUDA(copy(t1, x), "conv_run");
            const Op seq[5] = {{OpKind::Fwd3D, t1, nullptr, 0, 0, 0, 0},
                               {OpKind::DataReal, t1, A, num, B, 0, 0},
                               {OpKind::Bwd3D, t1, nullptr, 0, 0, 0, 0},
                               {OpKind::Merge, t1, x, num, 1, coef.a1, coef.b1},
                               {OpKind::Space, t1, S, num, B, 0, 0}};
            for (const Op& op : seq)
                if ((r = exec_op(c, op))) return r;
            CPRA_CHECK_CUDA(copy(x, t1), "conv_run");
        }
        return CPRA_B200_OK;
    };
    r = run_maybe_graph(c,
                        graph_key("conv_run", x, A, S, iters, b, final_step, want_err, c->space_mode, c->data_mode,
                                  c->fusion, c->fused3d),
                        enqueue);
    if (r) return r;
    if (want_err) {
        CPRA_CHECK_CUDA(cudaStreamSynchronize(c->stream), "conv_run");
        for (uint64_t i = 0; i < B; ++i) {
            const double v = std::sqrt(c->host_sums[2 * i]) / std::sqrt(c->host_sums[2 * i + 1]);
            if (c->dbl)
                static_cast<double*>(err_host)[i] = v;
            else
                static_cast<float*>(err_host)[i] = (float)v;
        }
    }
    return CPRA_B200_OK;
}

int cpra_b200_conv_run(cpra_b200_ctx* c, void* x, const void* A, const void* S, int iters, double beta,
                       int final_step, void* err_host) {
    CTX_OR_RETURN(c);
    return conv_run_impl(c, x, A, S, iters, beta, final_step, err_host);
}

// ---- raw-file I/O (include/detail/CPRA.inl:8-48; src/CPRA_MKL.cpp:156-225) ---
// Files hold elements of T back to back, no header.  Copies between a file and
// memory (device, managed or host) go through two pinned chunks on the copy
// stream: the file side of one chunk overlaps the copy of the other.  These
// helpers report errors through `msg` only, so that cpra_b200_cpra_files'
// writer thread can use them.

int io_prepare(cpra_b200_ctx* c) {
    if (!c->copy_stream)
        CPRA_CHECK_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!c->io_ready) CPRA_CHECK_CUDA(cudaEventCreateWithFlags(&c->io_ready, cudaEventDisableTiming), "cudaEventCreate");
    for (int k = 0; k < 2; ++k) {
        if (!c->io_ev[k])
            CPRA_CHECK_CUDA(cudaEventCreateWithFlags(&c->io_ev[k], cudaEventDisableTiming), "cudaEventCreate");
        if (c->io_pinned_bytes != c->io_chunk && c->io_pinned[k]) {
            cudaFreeHost(c->io_pinned[k]);
            c->io_pinned[k] = nullptr;
        }
        if (!c->io_pinned[k]) CPRA_CHECK_CUDA(cudaMallocHost(&c->io_pinned[k], c->io_chunk), "cudaMallocHost(io)");
    }
    c->io_pinned_bytes = c->io_chunk;
    return CPRA_B200_OK;
}

// copy_stream waits for the work already on the context's stream
int io_after_stream(cpra_b200_ctx* c) {
    CPRA_CHECK_CUDA(cudaEventRecord(c->io_ready, c->stream), "cudaEventRecord");
    CPRA_CHECK_CUDA(cudaStreamWaitEvent(c->copy_stream, c->io_ready, 0), "cudaStreamWaitEvent");
    return CPRA_B200_OK;
}

int file_to_mem(cpra_b200_ctx* c, FILE* f, char* dst, uint64_t bytes, std::string& msg) {
    bool used[2] = {false, false};
    uint64_t off = 0;
    cudaError_t e = cudaSuccess;
    for (int k = 0; off < bytes && e == cudaSuccess; k ^= 1) {
        const uint64_t len = std::min(c->io_chunk, bytes - off);
        if (used[k] && (e = cudaEventSynchronize(c->io_ev[k])) != cudaSuccess) break;
        if (std::fread(c->io_pinned[k], 1, len, f) != len) {
            cudaStreamSynchronize(c->copy_stream);
            msg = "short file: fewer bytes than the requested elements";
            return CPRA_B200_EARG;
        }
        if ((e = cudaMemcpyAsync(dst + off, c->io_pinned[k], len, cudaMemcpyDefault, c->copy_stream)) != cudaSuccess)
            break;
        e = cudaEventRecord(c->io_ev[k], c->copy_stream);
        used[k] = true;
        off += len;
    }
    const cudaError_t es = cudaStreamSynchronize(c->copy_stream);
    if (e == cudaSuccess) e = es;
    if (e != cudaSuccess) {
        msg = std::string("file read copy: ") + cudaGetErrorString(e);
        return CPRA_B200_ECUDA;
    }
    return CPRA_B200_OK;
}

int mem_to_file(cpra_b200_ctx* c, const char* src, uint64_t bytes, FILE* f, std::string& msg) {
    uint64_t issued = 0, written = 0, pend[2] = {0, 0};
    cudaError_t e = cudaSuccess;
    auto issue = [&](int k) {
        pend[k] = std::min(c->io_chunk, bytes - issued);
        e = cudaMemcpyAsync(c->io_pinned[k], src + issued, pend[k], cudaMemcpyDefault, c->copy_stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->io_ev[k], c->copy_stream);
        issued += pend[k];
    };
    for (int k = 0; k < 2 && issued < bytes && e == cudaSuccess; ++k) issue(k);
    for (int k = 0; written < bytes && e == cudaSuccess; k ^= 1) {
        if ((e = cudaEventSynchronize(c->io_ev[k])) != cudaSuccess) break;
        if (std::fwrite(c->io_pinned[k], 1, pend[k], f) != pend[k]) {
            cudaStreamSynchronize(c->copy_stream);
            msg = "file write failed";
            return CPRA_B200_EARG;
        }
        written += pend[k];
        if (issued < bytes) issue(k);
    }
    const cudaError_t es = cudaStreamSynchronize(c->copy_stream);
    if (e == cudaSuccess) e = es;
    if (e != cudaSuccess) {
        msg = std::string("file write copy: ") + cudaGetErrorString(e);
        return CPRA_B200_ECUDA;
    }
    return CPRA_B200_OK;
}

// `path` <- `bytes` of memory; the file is created or overwritten
int write_file(cpra_b200_ctx* c, const std::string& path, const void* src, uint64_t bytes, bool host, std::string& msg) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        msg = "cannot open " + path + " for writing";
        return CPRA_B200_EARG;
    }
    int r = CPRA_B200_OK;
    if (host) {
        if (std::fwrite(src, 1, bytes, f) != bytes) {
            msg = "file write failed: " + path;
            r = CPRA_B200_EARG;
        }
    } else {
        r = mem_to_file(c, static_cast<const char*>(src), bytes, f, msg);
    }
    if (std::fclose(f) != 0 && !r) {
        msg = "file close failed: " + path;
        r = CPRA_B200_EARG;
    }
    return r;
}

// the output files of starts [0, count) of x's gathered real parts (dev,
// [count][P][MN] of T) and of their errors (err [P][B] of T, host; may be
// null): <recon>.<index + i> and <errp>.<index + i>
int write_start_files(cpra_b200_ctx* c, const char* dev, const void* err, uint64_t P, uint64_t B, uint64_t count,
                      uint64_t elems_per_start, const std::string& recon, const std::string& errp, uint64_t index,
                      std::string& msg) {
    const uint64_t es = c->esize(), per = elems_per_start * es;
    std::vector<char> e(P * es);
    for (uint64_t i = 0; i < count; ++i) {
        const std::string sfx = "." + std::to_string(index + i);
        int r = write_file(c, recon + sfx, dev + i * per, per, false, msg);
        if (r) return r;
        if (!err) continue;
        // src/CPRA_MKL.cpp:195-196: per_error[p] = error[p * n + i]
        for (uint64_t p = 0; p < P; ++p)
            std::memcpy(e.data() + p * es, static_cast<const char*>(err) + (p * B + i) * es, es);
        if ((r = write_file(c, errp + sfx, e.data(), P * es, true, msg))) return r;
    }
    return CPRA_B200_OK;
}

int cpra_b200_read_matrix(cpra_b200_ctx* c, const char* path, void* dst, uint64_t count, uint64_t elem_bytes) {
    CTX_OR_RETURN(c);
    if (!path || !dst) return fail(CPRA_B200_EARG, "read_matrix: null pointer");
    // include/detail/CPRA.inl:11-21: a missing file and a zero size are errors
    if (count == 0 || elem_bytes == 0) return fail(CPRA_B200_EARG, "read_matrix: zero size");
    int r = flush(c);
    if (r) return take_deferred(c);
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(CPRA_B200_EARG, std::string("read_matrix: cannot open ") + path);
    std::string msg;
    r = io_prepare(c);
    if (!r) r = io_after_stream(c);
    if (!r) r = file_to_mem(c, f, static_cast<char*>(dst), count * elem_bytes, msg);
    std::fclose(f);
    if (r && !msg.empty()) return fail(r, "read_matrix: " + msg + " (" + path + ")");
    return r;
}

int cpra_b200_write_matrix(cpra_b200_ctx* c, const char* path, const void* src, uint64_t count, uint64_t elem_bytes) {
    CTX_OR_RETURN(c);
    if (!path || !src) return fail(CPRA_B200_EARG, "write_matrix: null pointer");
    if (count == 0 || elem_bytes == 0) return fail(CPRA_B200_EARG, "write_matrix: zero size");  // CPRA.inl:39-43
    int r = flush(c);
    if (r) return take_deferred(c);
    std::string msg;
    r = io_prepare(c);
    if (!r) r = io_after_stream(c);
    if (!r) r = write_file(c, path, src, count * elem_bytes, false, msg);
    if (r && !msg.empty()) return fail(r, "write_matrix: " + msg);
    return r;
}

int cpra_b200_write_starts(cpra_b200_ctx* c, const char* recon_prefix, const char* err_prefix, uint64_t file_index,
                           const void* x, const void* err_host, uint64_t P, uint64_t batch, uint64_t count) {
    CTX_OR_RETURN(c);
    if (!recon_prefix || !x) return fail(CPRA_B200_EARG, "write_starts: null pointer");
    if (P == 0 || batch == 0 || count == 0 || count > batch)
        return fail(CPRA_B200_EARG, "write_starts: P, batch >= 1 and 1 <= count <= batch");
    if ((err_prefix == nullptr) != (err_host == nullptr))
        return fail(CPRA_B200_EARG, "write_starts: err_prefix and err_host go together");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t MN = c->plane();
    if ((r = ensure_buffer(c, &c->io_dev, &c->io_dev_bytes, count * P * MN * c->esize(), "cudaMalloc(io)"))) return r;
    if ((r = io_prepare(c))) return r;
    CPRA_CHECK_CUDA(launch_real_starts(c->dbl, x, c->io_dev, MN, P, batch, 0, count, c->stream), "write_starts");
    if ((r = io_after_stream(c))) return r;
    std::string msg;
    r = write_start_files(c, static_cast<const char*>(c->io_dev), err_host, P, batch, count, P * MN, recon_prefix,
                          err_prefix ? err_prefix : "", file_index, msg);
    if (r) return fail(r, "write_starts: " + msg);
    return CPRA_B200_OK;
}

int cpra_b200_cpra_files(cpra_b200_ctx* c, const char* a_path, const char* s_path, const char* recon_prefix,
                         const char* err_prefix, uint64_t P, uint64_t total, int epi, int iters, int pre_iter,
                         double beta) {
    CTX_OR_RETURN(c);
    if (!a_path || !s_path || !recon_prefix || !err_prefix) return fail(CPRA_B200_EARG, "cpra_files: null pointer");
    if (P < 2) return fail(CPRA_B200_EARG, "cpra_files: P >= 2");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t MN = c->plane(), B = c->batch, es = c->esize();
    // src/CPRA_MKL.cpp:160-170: the modulus and support planes [P][m][n]
    if ((r = ensure_buffer(c, &c->io_A, &c->io_A_bytes, P * MN * es, "cudaMalloc(io A)"))) return r;
    if ((r = ensure_buffer(c, &c->io_S, &c->io_S_bytes, P * MN * es, "cudaMalloc(io S)"))) return r;
    if ((r = ensure_buffer(c, &c->io_x, &c->io_x_bytes, P * B * MN * c->csize(), "cudaMalloc(io x)"))) return r;
    if ((r = ensure_buffer(c, &c->io_dev, &c->io_dev_bytes, B * P * MN * es, "cudaMalloc(io)"))) return r;
    if ((r = cpra_b200_read_matrix(c, a_path, c->io_A, P * MN, es))) return r;
    if ((r = cpra_b200_read_matrix(c, s_path, c->io_S, P * MN, es))) return r;
    // :172-224: N = max(batch, total) starts in batches of the context's
    // batch size; a last partial batch runs whole and writes its first n
    const uint64_t N = std::max<uint64_t>(B, total);
    const bool with_err = epi > 0 && iters >= 1;
    std::vector<char> err[2] = {std::vector<char>(P * B * es, 0), std::vector<char>(P * B * es, 0)};
    std::thread writer;
    int wr = CPRA_B200_OK;
    std::string wmsg;
    auto join = [&]() {
        if (writer.joinable()) writer.join();
        return wr;
    };
    uint64_t file_index = 1;
    int k = 0;
    for (uint64_t left = N; left > 0; k ^= 1) {
        const uint64_t n = std::min(left, B);
        r = cpra_b200_initialize(c, c->io_x, P * B * MN * 2);
        if (!r)
            r = cpra_run_impl(c, c->io_x, c->io_A, c->io_S, P, B, epi, iters, pre_iter, beta, 1,
                              with_err ? err[k].data() : nullptr, nullptr, nullptr);
        // the previous batch's files were written while this batch computed
        if (join() && !r) r = fail(wr, "cpra_files: " + wmsg);
        if (r) return r;
        CPRA_CHECK_CUDA(launch_real_starts(c->dbl, c->io_x, c->io_dev, MN, P, B, 0, n, c->stream), "cpra_files");
        if ((r = io_prepare(c)) || (r = io_after_stream(c))) return r;
        writer = std::thread([c, n, P, B, MN, file_index, &err, k, &wr, &wmsg, recon = std::string(recon_prefix),
                              errp = std::string(err_prefix)]() {
            wr = write_start_files(c, static_cast<const char*>(c->io_dev), err[k].data(), P, B, n, P * MN, recon,
                                   errp, file_index, wmsg);
        });
        file_index += n;
        left -= n;
    }
    if (join()) return fail(wr, "cpra_files: " + wmsg);
    return CPRA_B200_OK;
}

int cpra_b200_conv_files(cpra_b200_ctx* c, const char* a_path, const char* s_path, const char* recon_prefix,
                         const char* err_prefix, uint64_t total, int iters, double beta) {
    CTX_OR_RETURN(c);
    if (!a_path || !s_path || !recon_prefix || !err_prefix) return fail(CPRA_B200_EARG, "conv_files: null pointer");
    int r = flush(c);
    if (r) return take_deferred(c);
    const uint64_t vol = c->plane() * c->l, B = c->batch, es = c->esize();
    // src/CONV_MKL.cpp:108-118: the modulus and support volumes [l][m][n]
    if ((r = ensure_buffer(c, &c->io_A, &c->io_A_bytes, vol * es, "cudaMalloc(io A)"))) return r;
    if ((r = ensure_buffer(c, &c->io_S, &c->io_S_bytes, vol * es, "cudaMalloc(io S)"))) return r;
    if ((r = ensure_buffer(c, &c->io_x, &c->io_x_bytes, B * vol * c->csize(), "cudaMalloc(io x)"))) return r;
    if ((r = ensure_buffer(c, &c->io_dev, &c->io_dev_bytes, B * vol * es, "cudaMalloc(io)"))) return r;
    if ((r = cpra_b200_read_matrix(c, a_path, c->io_A, vol, es))) return r;
    if ((r = cpra_b200_read_matrix(c, s_path, c->io_S, vol, es))) return r;
    // :119-165: max(batch, total) starts in batches; each start's volume
    // (real parts) and error to <prefix>.<k>, k counting starts from 1
    const uint64_t N = std::max<uint64_t>(B, total);
    const bool with_err = iters >= 1;
    std::vector<char> err[2] = {std::vector<char>(B * es, 0), std::vector<char>(B * es, 0)};
    std::thread writer;
    int wr = CPRA_B200_OK;
    std::string wmsg;
    auto join = [&]() {
        if (writer.joinable()) writer.join();
        return wr;
    };
    uint64_t file_index = 1;
    int k = 0;
    for (uint64_t left = N; left > 0; k ^= 1) {
        const uint64_t n = std::min(left, B);
        r = cpra_b200_initialize(c, c->io_x, B * vol * 2);
        if (!r) r = conv_run_impl(c, c->io_x, c->io_A, c->io_S, iters, beta, 1, with_err ? err[k].data() : nullptr);
        if (join() && !r) r = fail(wr, "conv_files: " + wmsg);
        if (r) return r;
        CPRA_CHECK_CUDA(launch_real_starts(c->dbl, c->io_x, c->io_dev, vol, 1, B, 0, n, c->stream), "conv_files");
        if ((r = io_prepare(c)) || (r = io_after_stream(c))) return r;
        writer = std::thread([c, n, B, vol, file_index, &err, k, &wr, &wmsg, recon = std::string(recon_prefix),
                              errp = std::string(err_prefix)]() {
            wr = write_start_files(c, static_cast<const char*>(c->io_dev), err[k].data(), 1, B, n, vol, recon, errp,
                                   file_index, wmsg);
        });
        file_index += n;
        left -= n;
    }
    if (join()) return fail(wr, "conv_files: " + wmsg);
    return CPRA_B200_OK;
}
}  // extern "C"
