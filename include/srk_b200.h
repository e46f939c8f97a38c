/*
 * srk_b200.h — C ABI of the B200 (sm_100a) resist-shrinkage operator library.
 *
 *   h = c * ( conv(Gx, g) * df/dx + conv(Gy, g) * df/dy )      (valid, W = N - 2*erosion)
 *
 * Every buffer is a device pointer; every image is column-major
 * buf[col*H + row] with batch stride N*N (inputs) or W*W (outputs).  Kernel
 * spectra are accepted in the reference's layout: the unnormalised R2C
 * spectrum of the fftshifted, column-major M x M padded kernel,
 * freq[kx*(M/2+1) + ky] (complex64 = two floats), M = the plan's spectra_M.
 *
 * All entry points are stream-ordered and asynchronous (no host sync); they
 * return a status instead of aborting.  The *_sync variants add a
 * cudaStreamSynchronize, like the reference's operators.
 *
 * The plan (srk_plan) replaces the reference's workspace structs
 * (SrkTrainWorkspace, SrkConvWorkspace, SrkAdjWorkspace, SrkTanWorkspace,
 * SrkTanAdjWorkspace): it owns the scratch, the re-laid-out kernel spectra
 * and the tile configuration.  A plan is bound to one device and must not be
 * used from two host threads at once.
 */
#ifndef SRK_B200_H
#define SRK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* srk_stream_t; /* == cudaStream_t */
typedef struct srk_plan_s* srk_plan;

typedef enum srk_status {
  SRK_OK = 0,
  SRK_ERR_INVALID_ARG = 1, /* bad size / null pointer / mismatch with the plan */
  SRK_ERR_UNSUPPORTED = 2, /* valid request the library cannot serve (e.g. tile too small) */
  SRK_ERR_ALLOC = 3,       /* device allocation failed */
  SRK_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
  SRK_ERR_CUDA = 5         /* a CUDA runtime call failed */
} srk_status;

typedef enum srk_dtype { SRK_F32 = 0, SRK_F16 = 1, SRK_BF16 = 2 } srk_dtype;

/* How the adjoint with respect to the convolved field applies the kernel.
 * SRK_ADJ_REFERENCE multiplies by the stored spectrum, i.e. convolves the
 * cotangent with G exactly like adjointWrtE (adjoint/srk_adjoint.cuh:301-382).
 * SRK_ADJ_TRUE multiplies by its conjugate, i.e. correlates with G, which is
 * the exact adjoint of the forward convolution for any kernel.  The two agree
 * for even kernels and differ by a sign for the odd Green's tensor. */
typedef enum srk_adj_convention { SRK_ADJ_REFERENCE = 0, SRK_ADJ_TRUE = 1 } srk_adj_convention;

/* Kernel schedule of the convolution engine.  THREE_PASS (default): three
 * launches per chunk of work tiles with the intermediates in a device
 * scratch buffer; a call larger than the scratch cycles through a ring of
 * three scratch slots, the first and last passes on two plan-owned streams
 * and the middle pass on the caller's, so the passes of neighbouring chunks
 * run side by side (forked from and joined back into the caller's stream:
 * the call stays stream-ordered and graph-capturable).  PERSISTENT: one
 * launch per call; the column/row/column passes of every work tile run as
 * tickets of a queue with their
 * intermediates in an L2-resident ring (falls back to THREE_PASS when the
 * scratch holds fewer than three work tiles).  SRK_TILE_AUTOTUNE plans time
 * both and keep the faster. */
typedef enum srk_schedule {
  SRK_SCHEDULE_PERSISTENT = 0,
  SRK_SCHEDULE_THREE_PASS = 1,
  SRK_SCHEDULE_DIRECT = 2,
  SRK_SCHEDULE_TENSOR_ROWS = 3
} srk_schedule;
/* SRK_SCHEDULE_TENSOR_ROWS (FP16/BF16 storage plans at tile 512, erosion
 * 1..64): the three-pass schedule with its first two passes on the tensor
 * cores — the column transform as a DFT (tcgen05.mma against cos / -sin
 * tables; the column FFT where the tile origins are not on 8-row boundaries
 * or N % 8 != 0) and the convolution along x per frequency row as a banded
 * complex matrix product instead of the row FFT, spectral product and
 * inverse row FFT (FP16 operands: the column spectra are stored as FP16,
 * FP32 accumulation).  Used by the pair operators (training forward,
 * forward, the VJP's forward part); the tangent, the tangent-adjoint and
 * the adjoint-type pass run the three-pass FFT schedule on such a plan.
 * The plan allocates the FP16 spectra planes (1 MB per work tile of its
 * scratch) and the DFT tables (256 KB) when the schedule is set. */
/* SRK_SCHEDULE_DIRECT: the training forward and srk_forward run as a direct
 * convolution on the tensor cores (tcgen05.mma, FP32 accumulation; FP16/BF16
 * storage in one pass, FP32 storage in three passes over an exact FP16
 * hi + lo split) instead of FFTs: (128 + KW - 1) * KW * 2 multiply-adds per
 * output pixel, so it only pays for small kernels.  Needs erosion >= 1,
 * 2*erosion+1 <= 63 and N % 8 == 0; the other operators keep the
 * three-pass FFT schedule.  The counterpart of the reference's cuDNN
 * forward (training/srk_cudnn_forward.cuh:194-269); SRK_TILE_AUTOTUNE
 * times it against the FFT schedules where it applies. */

typedef struct srk_plan_info {
  int N, W, erosion, B_max, spectra_M;
  float dx;
  int tile_M;       /* FFT tile size of the forward geometry */
  int tile_stride;  /* valid outputs per tile per axis */
  int tiles;        /* tiles per axis, forward geometry */
  int tiles_adj;    /* tiles per axis, adjoint (full N x N output) geometry */
  int chunk_wt;     /* work tiles per scratch chunk */
  size_t scratch_bytes;
  srk_dtype dtype;
  int schedule;       /* srk_schedule */
  int last_launches;  /* kernel launches of the last engine call */
  int last_grid;      /* CTAs of the last persistent launch */
  int last_lag;       /* rounds between phases in the last persistent launch */
  int last_nslot;     /* scratch ring slots of the last persistent launch */
  unsigned long long last_spins; /* dependency polls that found work not ready (completed launches) */
} srk_plan_info;

/* ---- library ------------------------------------------------------------ */
int srk_version(void);
const char* srk_status_string(srk_status s);
/* Message of the last failing call on this host thread ("" if none). */
const char* srk_last_error(void);

/* ---- plans ----------------------------------------------------------------
 * N, W, erosion: image size, valid size, halo (W == N - 2*erosion).
 * dx: pixel pitch (the convolution is scaled by dx^2).
 * B_max: largest batch a call may pass.
 * spectra_M: FFT size of the caller's spectra (N for srkTrainingForward,
 *            the reference's M_TILE for the OaS operators).
 * tile_M: 0 = choose by a cost model, SRK_TILE_AUTOTUNE = time every
 *         (tile, schedule) candidate once per device and configuration
 *         (cached on disk, see srk_autotune), else 128, 256 or 512.
 * scratch_budget_bytes: 0 = default (8 GiB, at most 1/16 of the device
 *         memory, at least 256 MiB); the scratch holds the work tiles in
 *         flight (5.8 MB each at N = 512), never more than B_max needs.
 * The plan also holds 2 W^2 B_max floats for the intermediate of the VJP
 * and the tangent-adjoint (u*v between the FFT passes and the transposed
 * stencil): every device buffer an operator uses is allocated here (plus the
 * ragged / slab tile tables on a key's first call), none by an operator. */
srk_status srk_plan_create(srk_plan* plan, int N, int W, int erosion, float dx, int B_max, int spectra_M,
                           srk_dtype dtype, int tile_M, size_t scratch_budget_bytes);
srk_status srk_plan_destroy(srk_plan plan);
#define SRK_TILE_AUTOTUNE (-1)
/* Time every (tile size, schedule) candidate of the forward operator for this
 * configuration on synthetic device data (up to 512 images) and return the
 * fastest.  Results are cached per device name and configuration in the file
 * named by $SRK_TUNE_CACHE (default ~/.cache/srk_b200_tune.txt). */
srk_status srk_autotune(int N, int W, int erosion, float dx, int B, srk_dtype dtype, int* tile_M, int* schedule);
srk_status srk_plan_get_info(srk_plan plan, srk_plan_info* info);
srk_status srk_plan_set_adj_convention(srk_plan plan, srk_adj_convention conv);
srk_status srk_plan_set_schedule(srk_plan plan, srk_schedule schedule);
/* Persistent-schedule tuning: lag (rounds between the phases of a work
 * tile; 0 = derived from the grid), grid (CTAs; 0 = all that fit), prefetch
 * (1 = fetch the next ticket while running the current one). */
srk_status srk_plan_set_persistent(srk_plan plan, int lag, int grid, int prefetch);
/* Synchronise `stream` and report a device-side failure of the plan's last
 * persistent launch (SRK_ERR_TIMEOUT if a bounded wait gave up).  Operators
 * also report such a failure of the previous call once it has completed. */
srk_status srk_plan_sync(srk_plan plan, srk_stream_t stream);
/* Failure-path self test: one CTA waits, bounded by spin_limit polls, for a
 * counter that nothing increments.  Returns SRK_ERR_TIMEOUT when the wait
 * gave up as designed (the context stays usable), SRK_OK never. */
srk_status srk_debug_wait_selftest(srk_plan plan, unsigned long long spin_limit, srk_stream_t stream);

/* Import caller spectra (reference layout, size spectra_M).  Done implicitly
 * by the operators whenever they see spectrum pointers different from the
 * last imported ones; call it again after changing spectrum contents in
 * place. */
srk_status srk_plan_import_spectra(srk_plan plan, const void* d_Gx_freq, const void* d_Gy_freq,
                                   srk_stream_t stream);
/* Set the kernel from its spatial form: d_Kx, d_Ky column-major KW x KW
 * floats, KW <= 2*erosion+1.  Spectra pointers passed to later calls may
 * then be NULL. */
srk_status srk_plan_set_kernel(srk_plan plan, const float* d_Kx, const float* d_Ky, int KW,
                               srk_stream_t stream);

/* ---- kernel generation (FP64 on the device) --------------------------------
 * Green's tensor Gx = (gamma/2pi)(x/r)K1(gamma r)w(r), Gy likewise, radial
 * Blackman window of radius R_w, zero at r = 0; x = (i - KW/2)*dx.
 * Replaces make_kernel (training/main_cd_training.cu:40-77). */
srk_status srk_green_tensor(float* d_Kx, float* d_Ky, int KW, double gamma, double R_w, double dx,
                            srk_stream_t stream);
/* Spectrum of a spatial kernel at size M in the reference layout, computed in
 * FP64.  Replaces srkPrecomputeKernelFreq (srk_forward.cuh:154-203). */
srk_status srk_precompute_kernel_freq(const float* d_K, int KW, int M, void* d_freq, srk_stream_t stream);

/* ---- operators (reference parameter lists; the plan replaces `ws`) ------- */

/* srkTrainingForward (training/srk_training_forward.cuh:175-241):
 * R_b = dx^2 (conv(E_b,Gx) dI_b/dx + conv(E_b,Gy) dI_b/dy), b < B.
 * d_E, d_I [B][N][N]; d_R [B][W][W]; spectra [N][N/2+1] (spectra_M == N). */
srk_status srk_training_forward(const float* d_E, const float* d_I, const void* d_Gx_freq,
                                const void* d_Gy_freq, int N, int W, int erosion, float dx, int B,
                                srk_stream_t stream, float* d_R, srk_plan plan);
srk_status srk_training_forward_sync(const float* d_E, const float* d_I, const void* d_Gx_freq,
                                     const void* d_Gy_freq, int N, int W, int erosion, float dx, int B,
                                     srk_stream_t stream, float* d_R, srk_plan plan);

/* srkForwardOaS (srk_forward.cuh:468-501): one image; d_ux, d_uy optional
 * [W][W] outputs of dx^2 conv(E,Gx), dx^2 conv(E,Gy) (may be NULL). */
srk_status srk_forward_oas(const float* d_E, const float* d_I, const void* d_Gx_freq, const void* d_Gy_freq,
                           int N, int W, int erosion, float dx, srk_stream_t stream, float* d_R,
                           srk_plan plan, float* d_ux, float* d_uy);

/* adjointSRK (adjoint/srk_adjoint.cuh:402-425): given v = dL/dR and the
 * forward's ux, uy: dL/dI = Dx^T(ux v) + Dy^T(uy v), dL/dE = dx^2 (G (*) (v dI/dx) + ...)
 * (kernel applied per the plan's convention).  d_dLdI, d_dLdE [N][N]. */
srk_status srk_adjoint(const float* d_v, const float* d_ux, const float* d_uy, const float* d_I,
                       const void* d_Gx_freq, const void* d_Gy_freq, int N, int W, int erosion, float dx,
                       srk_stream_t stream, float* d_dLdI, float* d_dLdE, srk_plan plan);

/* shrinkageTangentOaS (tan_tanadj/srk_tangent.cuh:111-151): JVP dh [W][W]. */
srk_status srk_tangent(const float* d_f, const float* d_g, const float* d_df, const float* d_dg,
                       const void* d_Gx_freq, const void* d_Gy_freq, int N, int W, int erosion, float dx,
                       srk_stream_t stream, float* d_dh, srk_plan plan);

/* shrinkageTangentAdjointOaS (tan_tanadj/srk_tangent_adjoint.cuh:105-159):
 * d_dLam_f, d_dLam_g [N][N]. */
srk_status srk_tangent_adjoint(const float* d_f, const float* d_g, const float* d_df, const float* d_dg,
                               const float* d_lam_h, const float* d_dlam_h, const void* d_Gx_freq,
                               const void* d_Gy_freq, int N, int W, int erosion, float dx,
                               srk_stream_t stream, float* d_dLam_f, float* d_dLam_g, srk_plan plan);

/* ---- save-for-backward contract (no reference counterpart of this exact
 * signature; it recomputes conv(g,G) instead of taking ux, uy) ------------
 * forward: h = srk_forward_oas with E = g, I = f, batched.
 * vjp: (dL/df, dL/dg) from v = dL/dh and the saved f, g; B images. */
srk_status srk_forward(const float* d_f, const float* d_g, int B, srk_stream_t stream, float* d_h,
                       srk_plan plan);
srk_status srk_vjp(const float* d_v, const float* d_f, const float* d_g, int B, srk_stream_t stream,
                   float* d_dLdf, float* d_dLdg, srk_plan plan);
srk_status srk_jvp(const float* d_f, const float* d_g, const float* d_df, const float* d_dg, int B,
                   srk_stream_t stream, float* d_dh, srk_plan plan);

/* ---- ragged batches: B images of different sizes in one launch -----------
 * The reference runs one image per call (srkForwardOaS, adjointSRK,
 * shrinkageTangentOaS, shrinkageTangentAdjointOaS above); these forms take
 * B images whose sizes are given by Ns, a HOST array of B sizes with
 * 2*erosion+1 <= Ns[b] <= the plan's N, all with the plan's erosion, dx,
 * tile size and spectra.  Every buffer holds the images one after another,
 * column-major: N-sized buffers Ns[b]^2 elements per image, W-sized ones
 * (Ns[b] - 2*erosion)^2.  The tile tables are uploaded once per distinct Ns
 * (stream ordered); issue the ragged calls of one plan on one stream. */
srk_status srk_forward_oas_ragged(const float* d_E, const float* d_I, const void* d_Gx_freq,
                                  const void* d_Gy_freq, int B, const int* Ns, int erosion, float dx,
                                  srk_stream_t stream, float* d_R, srk_plan plan);
srk_status srk_adjoint_ragged(const float* d_v, const float* d_ux, const float* d_uy, const float* d_I,
                              const void* d_Gx_freq, const void* d_Gy_freq, int B, const int* Ns, int erosion,
                              float dx, srk_stream_t stream, float* d_dLdI, float* d_dLdE, srk_plan plan);
srk_status srk_tangent_ragged(const float* d_f, const float* d_g, const float* d_df, const float* d_dg,
                              const void* d_Gx_freq, const void* d_Gy_freq, int B, const int* Ns, int erosion,
                              float dx, srk_stream_t stream, float* d_dh, srk_plan plan);
srk_status srk_tangent_adjoint_ragged(const float* d_f, const float* d_g, const float* d_df, const float* d_dg,
                                      const float* d_lam_h, const float* d_dlam_h, const void* d_Gx_freq,
                                      const void* d_Gy_freq, int B, const int* Ns, int erosion, float dx,
                                      srk_stream_t stream, float* d_dLam_f, float* d_dLam_g, srk_plan plan);

/* ---- column slabs of one image ----------------------------------------------
 * One N x N image split by columns (contiguous runs in the column-major
 * layout), e.g. across GPUs.  These compute the output columns [c0, c1) of
 * srkForwardOaS / shrinkageTangentOaS (columns of the W x W output) or of
 * adjointSRK (columns of the N x N outputs).  Every pointer addresses column
 * c0 of its array; the buffer behind it must hold these columns (clipped to
 * the array):
 *   forward, tangent: N-sized inputs columns [c0, c1 + 2*erosion); R / dh [c0, c1).
 *   adjoint: v, ux, uy (W-sized) columns [c0 - 2*erosion, c1); I columns
 *            [c0 - erosion - 1, c1 + erosion + 1); dLdI, dLdE [c0, c1).
 *   tangent-adjoint (outputs: columns [c0, c1) of dLam_f, dLam_g): f, df
 *            [c0 - erosion - 1, c1 + erosion + 1); g, dg [r0, rE + 2*erosion);
 *            lam, dlam [min(c0 - 2*erosion, r0), max(c1, rE)), where
 *            r0 = max(c0 - erosion - 1, 0), r1 = min(c1 - erosion + 1, W),
 *            rE = min(r0 + T*S, W) with T = ceil((r1 - r0) / S) whole tiles
 *            of the plan's tile_stride S (the W-sized intermediate of the
 *            dL/df part is computed by whole tiles from r0).
 * c1 - c0 must be a multiple of the plan's tile_stride (srk_plan_get_info)
 * unless c1 is the last output column (W, or N for the adjoint-type
 * outputs).  The plan is one made for the whole image (N <= its N).  The
 * reference has no slab form; these replace srkForwardOaS
 * (srk_forward.cuh:468-501), shrinkageTangentOaS (srk_tangent.cuh:111-151),
 * adjointSRK (srk_adjoint.cuh:402-425) and shrinkageTangentAdjointOaS
 * (srk_tangent_adjoint.cuh:105-159) on one slab. */
srk_status srk_forward_oas_slab(const float* d_E, const float* d_I, const void* d_Gx_freq,
                                const void* d_Gy_freq, int N, int erosion, float dx, int c0, int c1,
                                srk_stream_t stream, float* d_R, srk_plan plan);
srk_status srk_tangent_slab(const float* d_f, const float* d_g, const float* d_df, const float* d_dg,
                            const void* d_Gx_freq, const void* d_Gy_freq, int N, int erosion, float dx,
                            int c0, int c1, srk_stream_t stream, float* d_dh, srk_plan plan);
srk_status srk_adjoint_slab(const float* d_v, const float* d_ux, const float* d_uy, const float* d_I,
                            const void* d_Gx_freq, const void* d_Gy_freq, int N, int erosion, float dx,
                            int c0, int c1, srk_stream_t stream, float* d_dLdI, float* d_dLdE,
                            srk_plan plan);
srk_status srk_tangent_adjoint_slab(const float* d_f, const float* d_g, const float* d_df, const float* d_dg,
                                    const float* d_lam_h, const float* d_dlam_h, const void* d_Gx_freq,
                                    const void* d_Gy_freq, int N, int erosion, float dx, int c0, int c1,
                                    srk_stream_t stream, float* d_dLam_f, float* d_dLam_g, srk_plan plan);

/* ---- synthetic inputs on the device -----------------------------------------
 * Gaussian random fields as GpGenerator (third_party/include/stTestCore/
 * gp_generator.h:95-254): white N(0,1) noise on the Np x Np grid (Np = next
 * power of two >= N) filtered by sqrt(FFT2(c)) of the periodic covariance
 * c(r) = exp(-r^2 / (2 ell^2)), cropped to the top-left N x N; d_out
 * [B][N][N].  minmax = 1 scales every image to [0, 1].  srk_grf draws the
 * noise with Philox4x32-10 keyed by seed + b (image b does not depend on B);
 * srk_grf_filter takes caller noise [B][Np][Np] (column-major) instead. */
srk_status srk_grf(int B, int N, double ell, unsigned long long seed, int minmax, srk_stream_t stream,
                   float* d_out);
srk_status srk_grf_filter(const float* d_noise, int B, int N, double ell, int minmax, srk_stream_t stream,
                          float* d_out);
/* Line/space patterns as gen_lns_vertical / gen_lns_horizontal
 * (third_party/src/patternUtil/test_pattern.cu:83-109): kinds is a HOST
 * array of B entries, 0 = vertical lines, 1 = horizontal; period_px 0 = 4 FWHM. */
srk_status srk_lns(int B, int N, const int* kinds, float sigma_px, float period_px, int num_nbrs,
                   srk_stream_t stream, float* d_out);

/* ---- critical dimension (CD) of line/space signals ------------------------
 * MeasureCD_Batched (third_party/src/metricUtil/cd_measure_util.cu:310-437)
 * in one kernel per signal: L-fold windowed-sinc upsampling (half width A),
 * sub-sample zero crossings, nearest crossing left of the centre and at or
 * right of it; d_left, d_right, d_cd [B] in input pixels, written on the
 * device (no host synchronisation).  Signals are d_sig [B][n], n <= 8192. */
srk_status srk_measure_cd(const float* d_sig, int B, int n, int L, int A, srk_stream_t stream, float* d_left,
                          float* d_right, float* d_cd);
/* CD of the centre line of E_crop + coeff*R (axis 0: centre row, axis 1:
 * centre column), E [B][N][N], R [B][W][W] from srk_training_forward: the
 * crop / apply_shrinkage / extract / measure sequence of
 * training/main_cd_training.cu:193-261 fused into the same kernel. */
srk_status srk_cd_after_shrinkage(const float* d_E, const float* d_R, int B, int N, int W, int erosion, float coeff,
                                  int axis, int L, int A, srk_stream_t stream, float* d_left, float* d_right,
                                  float* d_cd);
/* The same CD without the full operator: R is computed on the measured line
 * only, by direct convolution with the spatial kernels d_Kx, d_Ky
 * (column-major KW x KW, KW odd <= min(2*erosion+1, 129)) — the strip idea of
 * training/main_compare.cu:70-133.  Signal E + coeff*R with R from E and I
 * (the training forward has E = I); erosion >= 1. */
srk_status srk_cd_strip(const float* d_E, const float* d_I, const float* d_Kx, const float* d_Ky, int KW, int N,
                        int W, int erosion, float dx, int B, float coeff, int axis, int L, int A, srk_stream_t stream,
                        float* d_left, float* d_right, float* d_cd);

/* ---- training forward without any device allocation ---------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (code running inside another framework's memory pool or under a fixed
 * memory budget, plug-ins whose host owns every allocation, paths where an
 * allocation could synchronise the device): same arguments and result as
 * srk_training_forward, but no plan and no allocation of any kind — all
 * scratch lives in one 32 MiB array compiled into the library (held by every
 * GPU that loads it until the process exits).  N must be 128, 256 or 512 and
 * the spectra are at size N.  The first call on a device resolves the
 * array's device address; make it outside any stream capture.  All calls
 * share the array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised. */
srk_status srk_training_forward_noalloc(const float* d_E, const float* d_I, const void* d_Gx_freq,
                                        const void* d_Gy_freq, int N, int W, int erosion, float dx, int B,
                                        srk_stream_t stream, float* d_R);

/* ---- storage-typed forms ----------------------------------------------------
 * Same operators with every image / cotangent / output buffer in the plan's
 * storage type (SRK_F32: float, SRK_F16: IEEE half, SRK_BF16: bfloat16),
 * passed as void*.  Arithmetic is FP32 throughout (every butterfly, the
 * spectral products and the combine); kernel spectra and the intermediate
 * spectra stay FP32.  The float* entry points above require an SRK_F32 plan.
 * No counterpart in the reference (its operators are fp32 only). */
srk_status srk_training_forward_t(const void* d_E, const void* d_I, const void* d_Gx_freq, const void* d_Gy_freq,
                                  int N, int W, int erosion, float dx, int B, srk_stream_t stream, void* d_R,
                                  srk_plan plan);
srk_status srk_forward_oas_t(const void* d_E, const void* d_I, const void* d_Gx_freq, const void* d_Gy_freq, int N,
                             int W, int erosion, float dx, srk_stream_t stream, void* d_R, srk_plan plan, void* d_ux,
                             void* d_uy);
srk_status srk_adjoint_t(const void* d_v, const void* d_ux, const void* d_uy, const void* d_I, const void* d_Gx_freq,
                         const void* d_Gy_freq, int N, int W, int erosion, float dx, srk_stream_t stream,
                         void* d_dLdI, void* d_dLdE, srk_plan plan);
srk_status srk_tangent_t(const void* d_f, const void* d_g, const void* d_df, const void* d_dg, const void* d_Gx_freq,
                         const void* d_Gy_freq, int N, int W, int erosion, float dx, srk_stream_t stream, void* d_dh,
                         srk_plan plan);
srk_status srk_tangent_adjoint_t(const void* d_f, const void* d_g, const void* d_df, const void* d_dg,
                                 const void* d_lam_h, const void* d_dlam_h, const void* d_Gx_freq,
                                 const void* d_Gy_freq, int N, int W, int erosion, float dx, srk_stream_t stream,
                                 void* d_dLam_f, void* d_dLam_g, srk_plan plan);
srk_status srk_forward_t(const void* d_f, const void* d_g, int B, srk_stream_t stream, void* d_h, srk_plan plan);
srk_status srk_vjp_t(const void* d_v, const void* d_f, const void* d_g, int B, srk_stream_t stream, void* d_dLdf,
                     void* d_dLdg, srk_plan plan);
srk_status srk_jvp_t(const void* d_f, const void* d_g, const void* d_df, const void* d_dg, int B,
                     srk_stream_t stream, void* d_dh, srk_plan plan);

#ifdef __cplusplus
}
#endif
#endif /* SRK_B200_H */
