// Host-side interface between the C-ABI layer (capi.cu) and the kernel
// launchers (kernels_*.cu).  Every launcher enqueues on the given stream and
// returns a cudaError_t from cudaGetLastError(); argument validation happens in
// the C-ABI layer before any launcher is called.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

namespace cpra_b200 {

// Process-wide count of kernels this library has launched (every launcher
// calls count_launches after its launches; read by cpra_b200_kernels_launched).
void count_launches(uint64_t n = 1);
// Sets the calling thread's message returned by cpra_b200_last_error().
void set_last_error(const std::string& msg);

// ---- transforms (kernels_fft.cu) ---------------------------------------
// Shifted 2D transform of `batch` MxN planes in place:
//   forward : x <- s * D (.) FFT(D (.) x)
//   inverse : x <- D (.) (IFFT(s * D (.) x) * scale)
// with D = (-1)^(row+col) and s = (-1)^(M/2 + N/2), which equals
// fftshift o DFT o fftshift for even M, N.  `tw_m`, `tw_n` are device tables
// exp(-2 pi i t / M) and exp(-2 pi i t / N) in the element precision.
// `work` is a device buffer of at least batch*M*N elements, used only by the
// non-power-of-two path.
cudaError_t launch_fft2d(bool dbl, void* x, uint64_t M, uint64_t N, uint64_t batch, bool inverse, double scale,
                         const void* tw_m, const void* tw_n, void* work, cudaStream_t st);
// Shifted 3D transform of `batch` volumes laid out [L][M][N] (N fastest).
cudaError_t launch_fft3d(bool dbl, void* x, uint64_t M, uint64_t N, uint64_t L, uint64_t batch, bool inverse,
                         double scale, const void* tw_m, const void* tw_n, const void* tw_l, void* work,
                         cudaStream_t st);
// The benchmark's 3D step (src/benchmark_mkl.cpp:164-170), `iters` times:
// Forward3D; DataConstraint (complex C, plane M*N*L); Backward3D (scale);
// SpaceConstraint (S, plane M*N*L, space_mode) as five axis passes per
// iteration, same bits as the four per-operator calls.  Power-of-two sizes
// 2..1024 on every axis.
bool constraint3d_fused_supported(uint64_t M, uint64_t N, uint64_t L);
cudaError_t launch_constraint3d(bool dbl, void* x, const void* C, const void* S, uint64_t M, uint64_t N, uint64_t L,
                                uint64_t batch, int iters, int space_mode, double scale, const void* tw_m,
                                const void* tw_n, const void* tw_l, void* work, cudaStream_t st);
// True when the 2D shape runs as one CTA per plane (one HBM round trip).
bool fft2d_single_cta(bool dbl, uint64_t M, uint64_t N);
// True when a 1D length is supported at all by the transforms.
bool fft_length_supported(uint64_t L);

// ---- element-wise operators (kernels_ew.cu) ------------------------------
enum SpaceMode : int { SPACE_THRESHOLD = 0, SPACE_POSITIVE_SCALED = 1 };
enum DataMode : int { DATA_SKIP_ZERO = 0, DATA_ALWAYS = 1 };

cudaError_t launch_space_constraint(bool dbl, void* x, const void* s, uint64_t num, uint64_t plane, int mode,
                                    cudaStream_t st);
cudaError_t launch_data_constraint_real(bool dbl, void* x, const void* a, uint64_t num, uint64_t plane, int mode,
                                        cudaStream_t st);
cudaError_t launch_data_constraint_complex(bool dbl, void* x, const void* c, uint64_t num, uint64_t plane,
                                           cudaStream_t st);
cudaError_t launch_merge_add(bool dbl, const void* src, void* dst, double alpha, double beta, uint64_t num,
                             cudaStream_t st);
cudaError_t launch_scale(bool dbl, void* x, double factor, uint64_t num, cudaStream_t st);
cudaError_t launch_fftshift2d(bool dbl, void* x, uint64_t M, uint64_t N, uint64_t batch, cudaStream_t st);
cudaError_t launch_fftshift3d(bool dbl, void* x, uint64_t M, uint64_t N, uint64_t L, uint64_t batch,
                              cudaStream_t st);
cudaError_t launch_uniform(bool dbl, void* x, uint64_t num, uint64_t seed, uint64_t stream_id, cudaStream_t st);
// real parts of starts first..first+count-1 of x [P][B][MN], per start: dst [count][P][MN]
cudaError_t launch_real_starts(bool dbl, const void* x, void* dst, uint64_t MN, uint64_t P, uint64_t B, uint64_t first,
                               uint64_t count, cudaStream_t st);
// ||old_i|| and ||new_i|| over `span` elements at stride `stride` for i < batch,
// accumulated in double into sums[2*batch] (deterministic two-level reduction
// through `partials`, >= batch * CONVERGE_BLOCKS * 2 doubles).
constexpr int CONVERGE_BLOCKS = 64;
cudaError_t launch_norm_pairs(bool dbl, const void* a, const void* b, uint64_t span, uint64_t stride,
                              uint64_t batch, double* partials, double* sums, cudaStream_t st);
// stage 2 of the two-level reductions: sums[2b], sums[2b+1] from the
// CONVERGE_BLOCKS partial pairs of each of `batch` members, in index order
cudaError_t launch_norm_final(const double* partials, double* sums, uint64_t batch, cudaStream_t st);
// R-factor sums of `batch` centred spectra F (the Forward2D of each pattern):
// sums[2b] = sum_px | |F_b| - A_b |, sums[2b+1] = sum_px A_b, in double, with
// A_b = A + b * a_stride; deterministic two-level reduction through `partials`
// (>= batch * CONVERGE_BLOCKS * 2 doubles).
cudaError_t launch_rfactor_sums(bool dbl, const void* F, const void* A, uint64_t a_stride, uint64_t plane,
                                uint64_t batch, double* partials, double* sums, cudaStream_t st);
cudaError_t launch_real2d_to_3d(bool dbl, const void* src, void* dst, const void* angles, uint64_t m, uint64_t n,
                                uint64_t p, uint64_t l, cudaStream_t st);
// atab (may be null): scratch of angle_table_bytes(p) (angle_table.cuh); with
// it, and p <= ANGLE_TABLE_MAX, each voxel visits only the slices that can
// reach it
cudaError_t launch_complex2d_to_3d(bool dbl, const void* src, void* dst, const void* angles, uint64_t m,
                                   uint64_t n, uint64_t p, uint64_t l, void* atab, cudaStream_t st);

// ---- fused difference-map iterations (kernels_dm.cu) ---------------------
// Coefficients of the four MergeAddData calls of one iteration
// (dst = alpha*src + beta*dst), in call order.
struct DmCoef {
    double a1, b1;  // x  -> t1
    double a2, b2;  // x  -> t2
    double a3, b3;  // t1 -> x
    double a4, b4;  // t2 -> x
};
// Carousel mix applied to x before the first iteration (src/CPRA_MKL.cpp:64-76):
// MIX_FIRST x <- 0.5*next + 0.5*x; MIX_LAST x <- 0.5*prev + 0.5*x;
// MIX_MIDDLE x <- 0.5*prev + 0*x, then x <- 0.5*next + 1*x.
enum MixMode : int { MIX_NONE = 0, MIX_FIRST = 1, MIX_LAST = 2, MIX_MIDDLE = 3 };
struct DmArgs {
    void* x;
    void* t1;
    void* t2;
    const void* xprev = nullptr;  // neighbouring angles' planes for the mix
    const void* xnext = nullptr;
    int mix = MIX_NONE;
    int init_from_x = 0;  // t1 = t2 = x (after the mix) instead of the t1/t2 buffers' contents
    const void* A;       // modulus constraint plane(s)
    uint64_t a_stride;   // elements between consecutive patterns' planes (0: shared)
    const void* S;       // support plane(s)
    uint64_t s_stride;
    uint64_t M, N, batch;
    int iters;
    int space_mode;
    int data_mode;
    DmCoef c;
    uint64_t L = 1;  // 3D difference map: volumes [batch][L][M][N] (launch_dm3d_iterations)
    int tmem = 1;    // 128 x 128: x and t2 resident in tensor memory (k_dm_tm) instead of L2 (k_dm)
};
bool dm_fused_supported(bool dbl, uint64_t M, uint64_t N);
cudaError_t launch_dm_iterations(bool dbl, const DmArgs& a, const void* tw, cudaStream_t st);
// Resident CTAs of one angle's fused launch (k_dm: one per pattern) per SM,
// and the CTA count of that launch: how much of the GPU one angle fills.
int dm_fused_ctas_per_sm(uint64_t M);
// The difference-map iteration with the 3D transforms (src/CONV_MKL.cpp:37-88)
// on [batch][L][M][N] volumes, A and S one volume each (a_stride, s_stride
// unused), `iters` times as ten axis passes per iteration; same bits as the
// 12 operator calls.  Power-of-two sizes 2..1024 (constraint3d_fused_supported).
cudaError_t launch_dm3d_iterations(bool dbl, const DmArgs& a, double scale, const void* tw_m, const void* tw_n,
                                   const void* tw_l, void* work, cudaStream_t st);

// ---- the same iterations as line passes at 256 and 512 (kernels_dm_large.cu) ----
// Float square planes with the threshold SpaceConstraint; S shared
// (s_stride 0) or per pattern (s_stride M*N).  `scratch` holds
// dm_large_scratch_bytes (the row spectra of both halves and the support mask).
bool dm_large_supported(bool dbl, uint64_t M, uint64_t N, int space_mode);
uint64_t dm_large_scratch_bytes(uint64_t M, uint64_t N, uint64_t batch, uint64_t s_stride);
cudaError_t launch_dm_large(const DmArgs& a, const void* tw, void* scratch, cudaStream_t st);
// the row pass of one angle's large-plane iterations: CTAs per SM and per launch
int dm_large_ctas_per_sm(uint64_t M);
uint64_t dm_large_row_ctas(uint64_t M, uint64_t batch);

// ---- central slices and the amplitude-loss adjoints (kernels_adj.cu) --------
// Orientation table of P slices: sines and cosines of the tilts ang[p] and of
// the in-plane rotations rot[p] (rot may be null: none), orient_table_bytes.
uint64_t orient_table_bytes(bool dbl, uint64_t p);
cudaError_t launch_orient_table(bool dbl, const void* ang, const void* rot, void* tab, uint64_t p, cudaStream_t st);
// slices out[p] ([P][N][M]) of the [L][N][M] volume V at the table's orientations
cudaError_t launch_slice(bool dbl, const void* V, const void* tab, void* out, uint64_t m, uint64_t n, uint64_t p,
                         uint64_t l, cudaStream_t st);
// G = dL/ds (scratch, [P][N][M]), gV = dL/dV, sums[3p] = loss of slice p,
// sums[3p+1] = dL/d ang[p], sums[3p+2] = dL/d rot[p] (partials: >= P *
// CONVERGE_BLOCKS * 3 doubles); ang orders the slices for the gather (atab)
cudaError_t launch_slice_loss_grad(bool dbl, const void* V, const void* ang, const void* tab, const void* A, void* G,
                                   void* gV, uint64_t m, uint64_t n, uint64_t p, uint64_t l, double* partials,
                                   double* sums, void* atab, cudaStream_t st);
// one Adam step (step >= 1) on the nv reals of V, the P tilts and (rot not
// null) the P rotations from gV and the per-slice sums; moments: 2 nv + 4 P
// elements, zero before step 1; loss <- sum_p sums[3p]
cudaError_t launch_refine_step(bool dbl, void* V, uint64_t nv, void* ang, void* rot, const void* gV, void* moments,
                               uint64_t P, const double* sums, double lr_volume, double lr_angle, double lr_rot,
                               int step, double* loss, cudaStream_t st);
// real volume <-> complex volume: to_complex: cplx = real + 0i; else real =
// Re(cplx) * scale (n values)
cudaError_t launch_real_complex(bool dbl, bool to_complex, void* real, void* cplx, double scale, uint64_t n,
                                cudaStream_t st);

// ---- fused HIO + shrinkwrap iterations (kernels_hio.cu) -----------------------
struct HioArgs {
    void* x;            // [batch][M][N] complex, in/out
    void* estimate;     // optional [batch][M][N] complex out: S (.) P_M(x) after the last iteration
    const void* A;      // modulus planes, pattern b at A + b*a_stride
    uint64_t a_stride;
    void* S;            // support planes (float, > 0.5 = inside), in/out, pattern b at S + b*s_stride
    uint64_t s_stride;
    const void* blur;   // [updates][M] Gaussian transfer tables (device), or null
    uint64_t M, N, batch;
    int iters, sw_every, positivity, data_mode;
    double beta, threshold;
    int tmem = 1;  // 128 x 128: the half of x that k_hio sends through L2 stays in tensor memory
    int* err = nullptr;  // cluster kernel: device word set to 1 when a wait for a peer's data ran out
    int withhold = 0;    // cluster kernel, failure test: the first CTA withholds its first blocks
};
bool hio_fused_supported(bool dbl, uint64_t M, uint64_t N);
cudaError_t launch_hio_iterations(bool dbl, const HioArgs& a, const void* tw, cudaStream_t st);

// ---- the same iteration with each pattern over a thread-block cluster (kernels_hio.cu) ----
// Float square planes: 128 with 2, 4 or 8 CTAs per pattern, 256 with 8 or 16.
// Same bits as the one-CTA kernel of the same line split (k_hio_tm at 128)
// for every cluster size.  No scratch.
bool hio_cluster_supported(bool dbl, uint64_t L, int cluster);
size_t hio_cluster_smem_bytes(uint64_t L, int cluster);
// clusters of that size resident at once on the current device (0: none)
int hio_cluster_max_active(uint64_t L, int cluster);
cudaError_t launch_hio_cluster(const HioArgs& a, int cluster, const void* tw, cudaStream_t st);

// ---- the same HIO iteration as line passes through L2 (kernels_large.cu) ----
// Float square planes of 256 or 512; patterns run in chunks of `chunk`, each
// chunk through all iterations.  Scratch, 16-byte aligned: Y (chunk planes,
// complex), V (chunk planes, float), vmax (chunk unsigned ints), mask (chunk
// planes of bits).
bool hio_large_supported(bool dbl, uint64_t M, uint64_t N);
cudaError_t launch_hio_large(const HioArgs& a, const void* tw, void* Y, void* V, unsigned int* vmax, uint32_t* mask,
                             uint64_t chunk, cudaStream_t st);

}  // namespace cpra_b200
