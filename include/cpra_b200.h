/*
 * cpra_b200.h - C ABI of the B200 backend for carousel phase retrieval.
 *
 * One entry point per virtual of the reference's operator interface
 * CPRA::CpraImpl<T> (include/CPRA_Impl.hpp:18-63), plus construction,
 * allocation and a few extensions.  Plain pointers and sizes only; no CUDA or
 * C++ types cross this boundary.  The C++ drop-in backend B200Impl<T>
 * (include/cpra_b200/B200_Impl.hpp) and the Python bindings both sit on it.
 *
 * Conventions (the reference's, include/CPRA_Impl.hpp):
 *  - Data pointers are device-accessible: memory from cpra_b200_alloc (managed
 *    by default, like the reference's CudaManagedAllocator,
 *    include/Allocator.hpp:36-52) or any device allocation.  Complex data is
 *    interleaved (re, im) in the context's element type.
 *  - Operators are asynchronous on the context's stream, except
 *    cpra_b200_converge_error (writes a host pointer) and cpra_b200_sync.
 *    Consecutive calls that form the reference's difference-map iteration
 *    (src/CPRA_MKL.cpp:94-110) may be held back and run as one fused launch;
 *    cpra_b200_sync, cpra_b200_memcpy, cpra_b200_converge_error and any call
 *    outside that pattern run everything held first.  Read results only after
 *    cpra_b200_sync (as the reference's drivers do before touching buffers).
 *  - Element-wise constraints broadcast their plane over the batch:
 *    element i uses constraint element i % (num / batch_size).
 *  - Return codes: CPRA_B200_OK, CPRA_B200_EARG for argument errors (the
 *    reference returns false, include/detail/MKL_Impl.inl:11,34,55,73,89,112),
 *    CPRA_B200_ECUDA for CUDA runtime failures (the reference throws
 *    CPRA::cuda_error, include/CUDA_Error_Check.hpp:29-82), CPRA_B200_EUNSUP
 *    for shapes this backend does not implement.  cpra_b200_last_error()
 *    returns the calling thread's last message.
 *  - A context is not thread-safe (neither is the reference's,
 *    include/CUDA_Impl.cuh:45-46): use one per host thread.
 */
#ifndef CPRA_B200_H
#define CPRA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CPRA_B200_OK 0
#define CPRA_B200_EARG 1
#define CPRA_B200_ECUDA 2
#define CPRA_B200_EUNSUP 3

#define CPRA_B200_F32 0
#define CPRA_B200_F64 1

/* options for cpra_b200_set_option */
#define CPRA_B200_OPT_FUSION 1     /* 1 (default): fuse recognised iterations; 0: run every call as it comes */
#define CPRA_B200_OPT_SPACE_MODE 2 /* 0 (default): MKL_Impl.inl:70-84 threshold; 1: CUDA_Impl_Kernel.cuh:16-28 */
#define CPRA_B200_OPT_DATA_MODE 3  /* 0 (default): MKL_Impl.inl:86-106 (A==0 unconstrained); 1: CUDA kernel */
#define CPRA_B200_OPT_SEED 4       /* seed of cpra_b200_initialize's counter-based stream */
#define CPRA_B200_OPT_KERNEL_TIMING 5 /* 1: bracket each fused launch with CUDA events (cpra_b200_kernel_timing) */
#define CPRA_B200_OPT_GRAPH 7      /* 1: cpra_b200_cpra_run, cpra_b200_conv_run and cpra_b200_hio_batched record
                                    their launches as a CUDA graph per distinct argument set and replay it on
                                    repeated calls */
#define CPRA_B200_OPT_HIO_CHUNK 6  /* patterns per chunk of the 256/512 HIO line passes (bounds their scratch,
                                    12.125 bytes per pixel); 0 (default): the whole batch */
#define CPRA_B200_OPT_LANES 8      /* streams of cpra_b200_cpra_run's wavefront schedule: angle p of episode e
                                    runs beside angle p-2 of episode e+1 (it only waits for angle p-1 of its
                                    episode and angle p+1 of the one before).  0 (default): enough to fill
                                    the GPU's resident CTA slots 1.5 times when one angle's launch fills less
                                    than all of them, else 1; 1: one stream, angle after angle; k <= 16: at
                                    most k streams.  Episodes are spread evenly (no more lanes than it takes
                                    to give each the busiest lane's episode count).  Same results in every
                                    case. */
#define CPRA_B200_MAX_LANES 16
#define CPRA_B200_OPT_IO_CHUNK 9   /* bytes of each of the two pinned staging chunks of the file I/O entries
                                    (default 64 MiB, at least 4096) */
#define CPRA_B200_OPT_AUTOTUNE 10  /* 1: with CPRA_B200_OPT_LANES 0, the first cpra_b200_cpra_run of each key
                                    (plane size, batch, angles, iterations, fusion and modes) measures the
                                    lane counts 1-4 and the automatic choice on a copy of x (min(epi, 4)
                                    episodes each; the copy is allocated for the duration) and keeps the
                                    fastest in the context's cache; later runs of that key use it, host-buffer
                                    runs only once it is cached.  No tuning during a stream capture or for
                                    epi < 2; if the copy cannot be allocated the key keeps the automatic
                                    choice.  0 (default): the automatic choice.  Same results either way.
                                    The same option also measures, once per shape and on copies of the
                                    inputs: for cpra_b200_constraint3d, fused axis passes against the
                                    operator kernels (one iteration each; CPRA_B200_OPT_FUSED3D is then
                                    ignored there); for cpra_b200_hio_shrinkwrap at 256 and 512 with
                                    CPRA_B200_OPT_HIO_CHUNK 0, the line passes' chunk among the whole batch,
                                    a half and a quarter (min(iters, 20) iterations each); for
                                    cpra_b200_hio_shrinkwrap at 128 with CPRA_B200_OPT_HIO_CLUSTER 1, one
                                    CTA per pattern against clusters of 2, 4 and 8.  No measurement
                                    during a stream capture or when the copy cannot be allocated. */
#define CPRA_B200_OPT_FUSED3D 12   /* 1: cpra_b200_constraint3d and the recognised 3D difference-map iteration
                                    run as fused axis passes (5 and 10 passes per iteration); 0 (default):
                                    as the operator kernels, measured faster on B200 (64^3 to 256^3).  Same
                                    results either way. */
#define CPRA_B200_OPT_TMEM 11      /* 1 (default): the fused 128 x 128 kernels keep their per-thread iterates
                                    in the SM's tensor memory for the whole launch (x and t2 of the
                                    difference map, x of HIO); 0: through L2 once per iteration.  The
                                    difference map gives the same results either way; HIO with 1 splits
                                    each line over 8 threads (4 with 0), as the 128 x 128 operator
                                    transforms do, and agrees with 0 to rounding, not bit for bit. */
#define CPRA_B200_OPT_FAILURE_TEST 14 /* test of the cluster kernel's bounded waits: 1 makes the next cluster
                                    HIO launch withhold one CTA's first row blocks, so that its peers'
                                    waits run out after a second; the launch is marked failed (the next
                                    cpra_b200_sync returns CPRA_B200_ECUDA), the context stays usable.
                                    Cleared by that launch. */
#define CPRA_B200_OPT_HIO_CLUSTER 13 /* cpra_b200_hio_shrinkwrap and cpra_b200_hio_batched: each pattern of
                                    side 128 or 256 spread over a thread-block cluster of this many CTAs
                                    (128: 2, 4 or 8; 256: 8 or 16), the plane exchanged between the CTAs'
                                    shared memories over the cluster network instead of through L2; other
                                    sides and unsupported sizes keep their kernels.  0: one CTA per pattern
                                    at 128, line passes at 256.  1 (default): automatic, the cluster kernel
                                    only for a batch too small to fill the device otherwise, the largest
                                    cluster (128: 8, 4 or 2; 256: 8) whose CTAs take one SM each and all
                                    fit at once, and at 128 only with CPRA_B200_OPT_TMEM 1; with
                                    CPRA_B200_OPT_AUTOTUNE, 128 x 128 calls measure one CTA per pattern
                                    against clusters of 2, 4 and 8 once per (batch, iterations) on copies
                                    of x and S.  At 128 the results are those of the tensor-memory kernel
                                    bit for bit; at 256 the same for 8 and 16, and within rounding of the
                                    line passes.  A cluster CTA that waits more than a second for its
                                    peers' data marks the launch failed: the next cpra_b200_sync returns
                                    CPRA_B200_ECUDA. */

typedef struct cpra_b200_ctx cpra_b200_ctx;

/* Replaces CudaImpl(m, n, l, batch_size) (include/CUDA_Impl.cuh:16-52) and the
 * factory case NewCpraImpl(IMPL_TYPE, m, n, l, batch) (include/Impl_Factory.hpp:14-30).
 * dtype: CPRA_B200_F32 or CPRA_B200_F64.  Binds the current CUDA device. */
int cpra_b200_create(cpra_b200_ctx** out, int dtype, uint64_t m, uint64_t n, uint64_t l, uint64_t batch_size);
/* Replaces ~CudaImpl (include/CUDA_Impl.cuh:105-112). */
int cpra_b200_destroy(cpra_b200_ctx* ctx);
const char* cpra_b200_last_error(void);
/* Number of kernels this library has launched in this process (all contexts). */
uint64_t cpra_b200_kernels_launched(void);
int cpra_b200_set_option(cpra_b200_ctx* ctx, int option, int64_t value);
/* Extension: reads an option back.  CPRA_B200_OPT_LANES reads the number of
 * lanes cpra_b200_cpra_run uses for the context's batch (the automatic choice
 * resolved, or with CPRA_B200_OPT_AUTOTUNE the last run's measured choice;
 * before the episode-count cap). */
int cpra_b200_get_option(cpra_b200_ctx* ctx, int option, int64_t* value);
/* The context's stream as a cudaStream_t (for interoperation). */
int cpra_b200_get_stream(cpra_b200_ctx* ctx, void** stream);

/* Replaces AllocatorInterface::allocate/deallocate for the CUDA backend
 * (include/Allocator.hpp:36-52 managed, :18-34 device). managed != 0 gives
 * host-accessible memory. */
int cpra_b200_alloc(cpra_b200_ctx* ctx, void** out, uint64_t bytes, int managed);
int cpra_b200_free(cpra_b200_ctx* ctx, void* ptr);

/* CpraImpl::Initialize (include/CPRA_Impl.hpp:23): num values uniform in [0, 1). */
int cpra_b200_initialize(cpra_b200_ctx* ctx, void* flat_data, uint64_t num);
/* CpraImpl::Forward2D / Backward2D (include/CPRA_Impl.hpp:25,27): fftshift, DFT
 * over the context's m x n planes (batch_size of them), fftshift; Backward2D
 * scales by 1/(m*n). */
int cpra_b200_forward2d(cpra_b200_ctx* ctx, void* flat_input);
int cpra_b200_backward2d(cpra_b200_ctx* ctx, void* flat_input);
/* CpraImpl::FFTShift2D (include/CPRA_Impl.hpp:29). */
int cpra_b200_fftshift2d(cpra_b200_ctx* ctx, void* flat_input, uint64_t M, uint64_t N, uint64_t batch);
/* CpraImpl::Forward3D / Backward3D (include/CPRA_Impl.hpp:31,33) on [l][m][n]
 * volumes; FFTShift3D (:35). */
int cpra_b200_forward3d(cpra_b200_ctx* ctx, void* flat_input);
int cpra_b200_backward3d(cpra_b200_ctx* ctx, void* flat_input);
int cpra_b200_fftshift3d(cpra_b200_ctx* ctx, void* flat_input, uint64_t M, uint64_t N, uint64_t L, uint64_t batch);
/* CpraImpl::SpaceConstraint (include/CPRA_Impl.hpp:37). */
int cpra_b200_space_constraint(cpra_b200_ctx* ctx, void* flat_src, const void* flat_constr, uint64_t num,
                               uint64_t batch_size);
/* CpraImpl::DataConstraint, real modulus overload (include/CPRA_Impl.hpp:39). */
int cpra_b200_data_constraint_real(cpra_b200_ctx* ctx, void* flat_src, const void* flat_constr, uint64_t num,
                                   uint64_t batch_size);
/* CpraImpl::DataConstraint, complex overload (include/CPRA_Impl.hpp:41). */
int cpra_b200_data_constraint_complex(cpra_b200_ctx* ctx, void* flat_src, const void* flat_constr, uint64_t num,
                                      uint64_t batch_size);
/* CpraImpl::MergeAddData (include/CPRA_Impl.hpp:45): dst = alpha*src + beta*dst.
 * alpha and beta are rounded to the context's element type. */
int cpra_b200_merge_add(cpra_b200_ctx* ctx, const void* flat_src, void* flat_dst, double alpha, double beta,
                        uint64_t num);
/* CpraImpl::Normalization (include/CPRA_Impl.hpp:48): x *= 1/norm. */
int cpra_b200_normalization(cpra_b200_ctx* ctx, void* flat_src, double norm, uint64_t num);
/* CpraImpl::Real2DTo3DInterpolation (include/CPRA_Impl.hpp:53). */
int cpra_b200_real2d_to_3d(cpra_b200_ctx* ctx, const void* flat_2d_src, void* flat_3d_dst, const void* angles,
                           uint64_t m, uint64_t n, uint64_t p, uint64_t l);
/* CpraImpl::Complex2DTo3DInterpolation (include/CPRA_Impl.hpp:54), a stub in
 * the reference; here the trilinear gather merge of complex central slices. */
int cpra_b200_complex2d_to_3d(cpra_b200_ctx* ctx, const void* flat_2d_src, void* flat_3d_dst, const void* angles,
                              uint64_t m, uint64_t n, uint64_t p, uint64_t l);
/* CpraImpl::ConvergeError (include/CPRA_Impl.hpp:56; CUDA_Impl.inl:145-172):
 * old <- new - old over m*n*l*batch elements, then err_host[i] =
 * ||old_i|| / ||new_i|| over the first m*n elements of member i.  err_host is a
 * host (or managed) pointer of the element type; the call is synchronous. */
int cpra_b200_converge_error(cpra_b200_ctx* ctx, void* flat_old, const void* flat_new, void* err_host, uint64_t m,
                             uint64_t n, uint64_t l, uint64_t batch_size);
/* CpraImpl::Memcpy (include/CPRA_Impl.hpp:58): asynchronous copy on the stream. */
int cpra_b200_memcpy(cpra_b200_ctx* ctx, void* dst, const void* src, uint64_t bytes);
/* CpraImpl::Sync (include/CPRA_Impl.hpp:60). */
int cpra_b200_sync(cpra_b200_ctx* ctx);

/* Extension: `iters` difference-map iterations of src/CPRA_MKL.cpp:94-110 in one
 * call, with the driver's coefficients derived from beta
 * (-1/beta, 1+1/beta), (1/beta, 1-1/beta), (beta, 1), (-beta, 1).  Pattern b of
 * the batch uses A + b*a_stride and S + b*s_stride (0: one shared plane, the
 * reference's broadcast).  x, t1, t2 hold `batch` m x n planes. */
int cpra_b200_dm_iterations(cpra_b200_ctx* ctx, void* x, void* t1, void* t2, const void* A, uint64_t a_stride,
                            const void* S, uint64_t s_stride, uint64_t batch, double beta, int iters);

/* Extension: the reference's carousel driver ShrinkWrap_CPRA_MKL_Sample
 * (src/CPRA_MKL.cpp:35-140) on `P` angles of `batch` starts each, x laid out
 * [P][batch][m][n] (the context's plane size; batch must equal the context's):
 *   pre_iter iterations on angle 0 (:35-55),
 *   epi episodes over the angles in Gauss-Seidel order with the carousel mix
 *   (:59-124), `iters` iterations per angle,
 *   and, if final_step != 0, the final projection of every angle (:126-140).
 * A and S hold one m x n plane per angle.  If err_host is not null it receives
 * the P*batch convergence errors of the last episode (:86-91,113-121, computed
 * as ConvergeError does); t1/t2/old are context-owned device buffers.
 * P >= 2 (the mix reads angles p-1 and p+1). */
int cpra_b200_cpra_run(cpra_b200_ctx* ctx, void* x, const void* A, const void* S, uint64_t P, uint64_t batch,
                       int epi, int iters, int pre_iter, double beta, int final_step, void* err_host);

/* Extension: the conventional 3D driver ShrinkWrap_CONV_MKL_Sample
 * (src/CONV_MKL.cpp:10-88) on the context's batch of [l][m][n] volumes x
 * (device), with one modulus volume A and one support volume S (broadcast
 * over the batch): t1 = t2 = x, `iters` difference-map iterations with
 * Forward3D/Backward3D (fused into axis passes for power-of-two volumes, else
 * the 12 operator calls), and, if final_step != 0, the final projection.  If
 * err_host is not null it receives the batch's convergence errors of the last
 * iteration, computed as ConvergeError does (CUDA_Impl.inl:145-172: over the
 * first m*n elements of each volume); the reference always computes them.
 * Results are those of the reference's call sequence on this backend.  With
 * err_host: synchronous; else asynchronous on the context's stream. */
int cpra_b200_conv_run(cpra_b200_ctx* ctx, void* x, const void* A, const void* S, int iters, double beta,
                       int final_step, void* err_host);

/* Extension: cpra_b200_cpra_run on HOST buffers (x, A, S laid out as above),
 * the whole ShrinkWrap_CPRA_MKL_Sample call of src/CPRA_MKL.cpp:35-140 with
 * its data in host memory, as the reference's caller holds it.  Angle p's
 * planes are uploaded on a context-owned copy stream and the first episode
 * waits for angle p+1 only before it runs angle p; with the final projection,
 * angle p's result is read back as soon as its projection is done.  x_host is
 * overwritten with the result.  Pinned host buffers make the copies overlap
 * the computation (pageable ones work, without overlap).  The device copies of
 * x, A and S are context-owned.  Synchronous; results are bit-identical to
 * cpra_b200_cpra_run on the same data. */
int cpra_b200_cpra_run_host(cpra_b200_ctx* ctx, void* x_host, const void* A_host, const void* S_host, uint64_t P,
                            uint64_t batch, int epi, int iters, int pre_iter, double beta, int final_step,
                            void* err_host);

/* Extension: the reference's raw-file reader Cpra::ReadMatrixFromFile
 * (include/detail/CPRA.inl:8-28), `count` elements of `elem_bytes` each, no
 * header, into dst (device, managed or host memory).  The file is read in
 * pinned chunks, each chunk's read overlapping the copy of the one before.
 * Errors, as the reference's: a missing file, a zero size; and a file shorter
 * than count elements (the reference's fread leaves the rest unwritten and
 * reports success).  Synchronous; ordered after the context's earlier work. */
int cpra_b200_read_matrix(cpra_b200_ctx* ctx, const char* path, void* dst, uint64_t count, uint64_t elem_bytes);

/* Extension: Cpra::WriteMatrixToFile (include/detail/CPRA.inl:30-48): `count`
 * elements of `elem_bytes` each from src (device, managed or host memory) to
 * a raw file, created or overwritten (the reference also prints a notice when
 * it overwrites), through the same pinned chunks.  Synchronous. */
int cpra_b200_write_matrix(cpra_b200_ctx* ctx, const char* path, const void* src, uint64_t count,
                           uint64_t elem_bytes);

/* Extension: the output files of src/CPRA_MKL.cpp:186-209 for starts
 * 0..count-1 of a carousel run x ([P][batch][m][n] complex T, device memory)
 * and its errors err_host ([P][batch] T, host memory, as cpra_b200_cpra_run
 * returns them): for start i,
 *   <recon_prefix>.<file_index + i>  the real parts of its P planes, [P][m][n] T;
 *   <err_prefix>.<file_index + i>    its P errors, P elements of T
 * (the reference writes sizeof(float)*P elements there, reading past its P
 * errors; here the file holds the P errors only).  The real parts are
 * gathered per start on the device, then streamed out through the pinned
 * chunks.  err_prefix and err_host both null: no error files.  Synchronous. */
int cpra_b200_write_starts(cpra_b200_ctx* ctx, const char* recon_prefix, const char* err_prefix, uint64_t file_index,
                           const void* x, const void* err_host, uint64_t P, uint64_t batch, uint64_t count);

/* Extension: the reference program's main loop (src/CPRA_MKL.cpp:156-225)
 * without its command-line parser: reads the modulus and support planes
 * ([P][m][n] T each) from a_path and s_path, then for max(batch, total)
 * starts in batches of the context's batch size: Initialize the guesses
 * ([P][batch][m][n], the context's seeded stream, one call per batch), run
 * cpra_b200_cpra_run (final projection on; errors when epi >= 1 and
 * iters >= 1, else zeros), and write each start's two files as
 * cpra_b200_write_starts does, numbered from 1 across batches.  A last
 * partial batch of n starts runs as a whole batch and writes its first n.
 * Each batch's files are written by a host thread while the next batch
 * computes.  Synchronous. */
int cpra_b200_cpra_files(cpra_b200_ctx* ctx, const char* a_path, const char* s_path, const char* recon_prefix,
                         const char* err_prefix, uint64_t P, uint64_t total, int epi, int iters, int pre_iter,
                         double beta);

/* Extension: the conventional program's main loop (src/CONV_MKL.cpp:103-172)
 * without its command-line parser: reads the modulus and support volumes
 * ([l][m][n] T each), then for max(batch, total) starts in batches of the
 * context's batch size: Initialize the guesses (one call per batch), run
 * cpra_b200_conv_run (final projection on; errors when iters >= 1, else
 * zeros), and write for each start k (from 1) <recon_prefix>.<k>, the real
 * parts of its volume, and <err_prefix>.<k>, its error (one element of T).
 * The reference writes one file per batch, holding only the batch's last
 * start, and stores every start's error into a one-element buffer
 * (:122, 141-146); here every start gets its own files.  Each batch's files
 * are written by a host thread while the next batch computes.  Synchronous. */
int cpra_b200_conv_files(cpra_b200_ctx* ctx, const char* a_path, const char* s_path, const char* recon_prefix,
                         const char* err_prefix, uint64_t total, int iters, double beta);

/* Extension (project-defined, no counterpart in the reference): R-factor of
 * `batch` patterns x ([batch][m][n], the context's plane size) against their
 * modulus planes A (pattern b uses A + b*a_stride; 0: one shared plane):
 *   r_host[b] = sum | |Forward2D(x_b)| - A_b | / sum A_b,
 * with |F| and both sums in double.  x is not modified.  Synchronous. */
int cpra_b200_rfactor(cpra_b200_ctx* ctx, const void* x, const void* A, uint64_t a_stride, uint64_t batch,
                      double* r_host);

/* Extension (project-defined, no counterpart in the reference): `iters`
 * hybrid input-output iterations with shrinkwrap, fused, for `batch` patterns
 * x ([batch][m][n] complex, in/out) with modulus planes A (pattern b at
 * A + b*a_stride) and supports S (float, > 0.5 = inside; in/out, pattern b at
 * S + b*s_stride).  With y = Backward2D(DataConstraint(Forward2D(x))):
 * x <- y inside the support (and Re y >= 0 if positivity != 0), else
 * x <- x - beta*y.  Every sw_every iterations (0: never) the support becomes
 * { v > threshold * max v }, v = |x| circularly blurred by a normalised
 * Gaussian whose sigma moves linearly from sigma_start (first update) to
 * sigma_end (last).  If estimate is not null it receives S (.) y of the final
 * x (the reconstruction).  Square float planes of 32, 64 or 128 run one CTA
 * per pattern, all iterations in one launch; 256 and 512 run two line passes
 * per iteration (columns with the modulus step; rows with the update and the
 * next forward row transform) over chunks of patterns
 * (CPRA_B200_OPT_HIO_CHUNK). */
int cpra_b200_hio_shrinkwrap(cpra_b200_ctx* ctx, void* x, const void* A, uint64_t a_stride, void* S,
                             uint64_t s_stride, uint64_t batch, int iters, double beta, int sw_every,
                             double sigma_start, double sigma_end, double threshold, int positivity,
                             void* estimate);

/* One size bucket of cpra_b200_hio_batched: `count` square side x side
 * patterns with x ([count][side][side] complex, in/out), A (modulus planes,
 * float), S (supports, float, in/out) and, optionally, the estimate output,
 * all contiguous per pattern (strides side*side). */
typedef struct cpra_b200_hio_bucket {
    uint64_t side;
    uint64_t count;
    void* x;
    const void* A;
    void* S;
    void* estimate;
    double sigma_start; /* this bucket's shrinkwrap blur schedule (pixels); <= 0: the call's */
    double sigma_end;
} cpra_b200_hio_bucket;
#define CPRA_B200_MAX_BUCKETS 64

/* Extension (project-defined, no counterpart in the reference): the HIO +
 * shrinkwrap iterations of cpra_b200_hio_shrinkwrap for patterns of uneven
 * sizes in one call: each bucket (side 32, 64, 128, 256 or 512; float
 * context) runs on its own stream, forked from and joined back into the
 * context's stream, so the buckets' launches overlap on the device.  The
 * context's m, n, batch do not constrain the buckets.  Asynchronous like the
 * other operators; same results per bucket as a cpra_b200_hio_shrinkwrap call
 * with that bucket's patterns. */
int cpra_b200_hio_batched(cpra_b200_ctx* ctx, const cpra_b200_hio_bucket* buckets, int n_buckets, int iters,
                          double beta, int sw_every, double sigma_start, double sigma_end, double threshold,
                          int positivity);

/* Extension: `iters` repetitions of the reference benchmark's 3D step
 * (src/benchmark_mkl.cpp:164-170) on the context's [batch][l][m][n] volumes:
 * Forward3D(x); DataConstraint(x, C, m*n*l*batch, batch) (complex C, one
 * volume shared by the batch); Backward3D(x); SpaceConstraint(x, S, same).
 * For power-of-two sizes (2..1024 per axis) an iteration is five axis passes
 * (the z pass runs forward transform, constraint and inverse transform per
 * line; the last x pass applies SpaceConstraint) with the same results, bit
 * for bit, as the four operator calls; other sizes run the four operators. */
int cpra_b200_constraint3d(cpra_b200_ctx* ctx, void* x, const void* C, const void* S, int iters);

/* Extension (project-defined): central slices of a Fourier volume.  V is
 * [l][n][m] complex (y fastest), slices are [p][n][m]; slice pixel (xIn, yIn)
 * at angle a (radians, element type) samples V bilinearly at z = l/2 - yr sin a,
 * x = xIn, y = m/2 - yr cos a, yr = m/2 - yIn (the merges' geometry); points
 * outside the volume read 0. */
int cpra_b200_slice(cpra_b200_ctx* ctx, const void* V, const void* angles, uint64_t m, uint64_t n, uint64_t p,
                    uint64_t l, void* slices);
/* Extension (project-defined): the amplitude loss L = sum (|slice(V, a_p)| - A_p)^2
 * (A: [p][n][m] element type) with its hand-written adjoints: grad_V (device,
 * [l][n][m] complex) receives dL/dRe V + i dL/dIm V, computed as the exact
 * transpose of the slice operator in gather form (deterministic);
 * grad_angles_host[p] (host, double, may be null) receives dL/da_p; loss_host
 * (double, may be null) receives L.  Sums are in double.  Synchronous. */
int cpra_b200_slice_loss_grad(cpra_b200_ctx* ctx, const void* V, const void* angles, const void* A, uint64_t m,
                              uint64_t n, uint64_t p, uint64_t l, void* grad_V, double* loss_host,
                              double* grad_angles_host);

/* Extension (project-defined): `steps` gradient-descent steps on the volume V
 * ([l][n][m] complex, device, in/out) and the angles (device, element type,
 * in/out) against the amplitude loss of cpra_b200_slice_loss_grad, with Adam
 * (Kingma & Ba 2015; beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected) and the
 * learning rates lr_volume, lr_angle.  Gradients come from the hand-written
 * adjoints each step (iterates are recomputed, not stored); the moments start
 * at zero each call.  loss_host (may be null) receives the loss before each
 * step; with it the call is synchronous. */
int cpra_b200_refine(cpra_b200_ctx* ctx, void* V, void* angles, const void* A, uint64_t m, uint64_t n, uint64_t p,
                     uint64_t l, int steps, double lr_volume, double lr_angle, double* loss_host);

/* Extension (project-defined): the slice operator with two orientation degrees
 * of freedom per slice: the tilt angles[p] as above and an in-plane rotation
 * rot[p] (radians, element type; may be null: none) of the detector grid.
 * Pixel (xIn, yIn) has xr = xIn - n/2, yr = m/2 - yIn, rotated to
 * xq = xr cos r - yr sin r, yq = xr sin r + yr cos r, and samples V
 * trilinearly at z = l/2 - yq sin a, x = n/2 + xq, y = m/2 - yq cos a (with
 * rot null this is cpra_b200_slice).  Coordinates and weights are computed in
 * the element type. */
int cpra_b200_slice_orient(cpra_b200_ctx* ctx, const void* V, const void* angles, const void* rot, uint64_t m,
                           uint64_t n, uint64_t p, uint64_t l, void* slices);
/* Extension (project-defined): cpra_b200_slice_loss_grad for the two-parameter
 * orientations; grad_rot_host[p] (host, double, may be null) receives
 * dL/drot_p.  Synchronous. */
int cpra_b200_slice_loss_grad_orient(cpra_b200_ctx* ctx, const void* V, const void* angles, const void* rot,
                                     const void* A, uint64_t m, uint64_t n, uint64_t p, uint64_t l, void* grad_V,
                                     double* loss_host, double* grad_angles_host, double* grad_rot_host);
/* Extension (project-defined): the amplitude loss of a real-space volume,
 * L = sum (|slice(Forward3D(vol), a_p, r_p)| - A_p)^2, and its gradients
 * through the hand-written adjoints of the modulus loss, the slice operator
 * and the transform: grad_vol (device, [l][n][m] element type) receives
 * dL/dvol = Re(Forward3D^H dL/dV), Forward3D^H being the inverse transform
 * without its 1/(m n l).  The context must have been created with this volume's
 * (m, n, l), powers of two 2..1024.  Synchronous. */
int cpra_b200_volume_loss_grad(cpra_b200_ctx* ctx, const void* vol, const void* angles, const void* rot,
                               const void* A, uint64_t m, uint64_t n, uint64_t p, uint64_t l, void* grad_vol,
                               double* loss_host, double* grad_angles_host, double* grad_rot_host);
/* Extension (project-defined): cpra_b200_refine for the two-parameter
 * orientations (rot may be null: not refined) and, with real_space != 0, a
 * real-space volume V ([l][n][m] element type) refined through
 * cpra_b200_volume_loss_grad's chain (the context then needs the volume's
 * (m, n, l)); with real_space == 0, V is the complex Fourier volume. */
int cpra_b200_refine_orient(cpra_b200_ctx* ctx, void* V, int real_space, void* angles, void* rot, const void* A,
                            uint64_t m, uint64_t n, uint64_t p, uint64_t l, int steps, double lr_volume,
                            double lr_angle, double lr_rot, double* loss_host);

/* Extension: the best of the random starts, the step the reference's
 * benchmark describes and omits (src/benchmark_mkl.cpp:127-138).  x is
 * [P][batch][m][n] (the driver's layout), A is [P][m][n].  The score of start
 * b is the mean over the P angles of its R-factor (cpra_b200_rfactor's
 * definition, float64); best_host receives the lowest-score start (the first
 * on ties), scores_host[batch] (may be null) the scores, and best_out (device
 * [P][m][n] complex, may be null) that start's planes.  Synchronous. */
int cpra_b200_best_start(cpra_b200_ctx* ctx, const void* x, const void* A, uint64_t P, uint64_t batch,
                         double* scores_host, uint64_t* best_host, void* best_out);

/* With CPRA_B200_OPT_KERNEL_TIMING on: total device time (ms) and number of
 * the fused difference-map launches since the last call, measured with CUDA
 * events on the context's stream; `pattern_iters` gets the patterns times
 * iterations they processed.  Synchronises the stream.  Resets the counters. */
int cpra_b200_kernel_timing(cpra_b200_ctx* ctx, double* ms, uint64_t* launches, uint64_t* pattern_iters);

/* ConvergeError for callers that cannot allocate GPU memory while they run
 * (device memory already reserved by another allocator or pool, loops that
 * must not be stalled by cudaFree's device-wide synchronisation, runs that must
 * not fail halfway on an allocation).  No counterpart in the reference: it is
 * the reference's ConvergeError (include/CPRA_Impl.hpp:56, CUDA_Impl.inl:145-172)
 * with the same result as cpra_b200_converge_error, but it needs no context and
 * calls no allocator: its partial sums live in a fixed scratch array compiled
 * into the library (a file-scope __device__ array of about 264 KiB that every
 * GPU loading the library holds until exit).  batch_size is limited to
 * CPRA_B200_NOALLOC_MAX_BATCH; larger batches are refused with CPRA_B200_EARG.
 * The scratch address is looked up on the first call made on each device, and
 * since CUDA loads a library's device code lazily, that call also places the
 * array in device memory: make it at start-up, before a memory pool reserves
 * the device and before any stream capture; later calls allocate nothing.  Do
 * not use the entry point across cudaDeviceReset.  All calls share the scratch:
 * calls that overlap on the GPU (other streams, other host threads) race.
 * dtype is CPRA_B200_F32 or CPRA_B200_F64; stream is a cudaStream_t (NULL: the
 * default stream); the call returns after err_host is written. */
#define CPRA_B200_NOALLOC_MAX_BATCH 256
int cpra_b200_converge_error_noalloc(int dtype, void* flat_old, const void* flat_new, void* err_host, uint64_t m,
                                     uint64_t n, uint64_t l, uint64_t batch_size, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CPRA_B200_H */
