// internal.h — private declarations shared by the library's translation
// units: status helpers, the plan object, and the engine launchers (one
// explicit instantiation per storage type lives in conv_<type>.cu so the
// kernel families compile in parallel).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <map>

#include "../../include/srk_b200.h"
#include "engine.cuh"

namespace srk {
// True while `s` is being captured into a CUDA graph: no event queries or
// host synchronisation may happen then.
inline bool stream_capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone;
}

inline thread_local std::string g_last_error;

inline srk_status fail(srk_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

inline srk_status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SRK_OK;
  // a failed allocation is not sticky: clear it so the next launch check
  // does not report it again
  if (e == cudaErrorMemoryAllocation) (void)cudaGetLastError();
  return fail(e == cudaErrorMemoryAllocation ? SRK_ERR_ALLOC : SRK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define SRK_TRY(expr)                        \
  do {                                       \
    const srk_status _s = (expr);            \
    if (_s != SRK_OK) return _s;             \
  } while (0)
#define SRK_CUDA(expr) SRK_TRY(cuda_status((expr), #expr))

}  // namespace srk

#ifndef SRK_RING
#define SRK_RING 3
#endif
struct srk_plan_s {
  int device = 0;
  int nsm = 0;  // SMs of the device (P1's L2 prefetch distance)
  int N = 0, W = 0, e = 0, B_max = 0, spectra_M = 0;
  float dx = 1.f;
  srk_dtype dtype = SRK_F32;
  srk_adj_convention conv = SRK_ADJ_REFERENCE;
  int M = 0, S = 0, T = 0, Ta = 0;
  int chunk = 0;
  float2* G[2] = {nullptr, nullptr};   // engine-layout spectra, scaled by dx^2/M^2
  bool have_G = false;
  const void* src[2] = {nullptr, nullptr};
  float2* tw = nullptr;                // W_M^m, float
  // spectrum import / set_kernel workspace, allocated with the plan so that
  // importing spectra needs no allocation and no host synchronisation:
  // FP64 twiddle tables at the tile size and at spectra_M, the column pass
  // of the kernel DFT (KW x M), the spatial recovery (spectra_M/2+1 x KW)
  // and one FP64 kernel (KW x KW), KW = 2*erosion+1
  double2* imp_tab = nullptr;          // (cos, sin)(2 pi m / M), m < M
  double2* imp_tabr = nullptr;         // the same at spectra_M
  double2* imp_P = nullptr;
  double2* imp_Tm = nullptr;
  double* imp_Kd = nullptr;
  // the bound kernels in space, FP64, on the full (2e+1)^2 support, centred
  // (recovered from the caller's spectra, or given to srk_plan_set_kernel)
  double* kd[2] = {nullptr, nullptr};
  // tensor-core direct schedule (direct.cu): FP16/BF16 band tables of the
  // bound kernels, a device error word written by its bounded waits
  uint16_t* direct_tabs = nullptr;
  bool direct_ready = false;
  unsigned int* direct_err = nullptr;  // [0] error word, [1] / [2] the direct / tensor-row tables' exponents
  // tensor-core row pass (hybrid.cu, SRK_SCHEDULE_TENSOR_ROWS): FP16 column
  // spectra planes of the chunks in flight, the band tables per ky, the FP64
  // row kernels they are made from
  __half* hyb_s1 = nullptr;
  size_t hyb_s1_bytes = 0;
  uint16_t* hyb_tabs = nullptr;
  double2* hyb_g = nullptr;
  unsigned int* hyb_mx = nullptr;  // largest |Z| per work tile in flight (float bits): the planes' scales
  void* p1g_tab = nullptr;         // column-DFT tables of the tensor-core column pass (storage type)
  bool hyb_ready = false;
  float2* scratch = nullptr;
  size_t scratch_bytes = 0;
  float* wbuf = nullptr;               // wx, wy for dL/df
  size_t wbuf_bytes = 0;
  int schedule = SRK_SCHEDULE_THREE_PASS;
  srk::Ctl* ctl = nullptr;             // persistent-kernel control block
  unsigned int* mailbox = nullptr;     // pinned host copy of (abort, where)
  cudaEvent_t mailbox_ev = nullptr;
  bool mailbox_pending = false;
  bool graph_mailbox = false;          // a captured persistent launch writes the mailbox on replay
  unsigned long long spin_limit = 1ull << 25;
  unsigned long long* mailbox_spins = nullptr;  // pinned: spin polls of the last launch
  int persist_lag = 0, persist_grid = 0, persist_prefetch = 0;
  int last_grid = 0, last_launches = 0, last_lag = 0, last_nslot = 0;
  // three-pass schedule over several chunks: a ring of kRing scratch slots,
  // P1 / P3 on streams of their own and P2 on the caller's, ordered per slot
  // by events, so the three phases of different chunks run side by side
  static constexpr int kRing = SRK_RING;
  cudaStream_t ps1 = nullptr, ps3 = nullptr;
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev1[kRing] = {}, ev2[kRing] = {}, ev3[kRing] = {};
  bool overlap = true;
  // ragged batches and column slabs: device tile tables (tile -> image,
  // per-image sizes/offsets), one set per key (the image sizes of a ragged
  // batch, or a slab's kind, image and columns), built on the first call
  // with that key and kept, so calls that alternate keys (a forward slab
  // and an adjoint slab of one training step) reuse them and can be
  // captured in a CUDA graph after one call of each outside the capture.
  struct TableSet {
    int4* tiles = nullptr;
    srk::RagImage* imgs = nullptr;
    int ntiles_fwd = 0, ntiles_adj = 0, nblk = 0;
    long long sum_nn = 0, sum_ww = 0;
    unsigned long long last_use = 0;
  };
  static constexpr size_t kMaxTableSets = 64;
  std::map<std::vector<int>, TableSet> tables;
  unsigned long long table_clock = 0;
  // the set selected by the current call
  int4* rag_tiles = nullptr;
  srk::RagImage* rag_imgs = nullptr;
  int rag_ntiles_fwd = 0, rag_ntiles_adj = 0, rag_nblk = 0;
  long long rag_sum_nn = 0, rag_sum_ww = 0;
};

namespace srk {

// Run one engine operator over all work tiles of geometry g (conv_<type>.cu).
template <int OP, typename T>
srk_status launch_conv(srk_plan_s* p, const OpArgs& a, const Geom& g, bool conjG, cudaStream_t s);

// Tensor-core direct convolution of the forward (direct.cu).
bool direct_supported(const srk_plan_s* p, int N, std::string* why);
size_t direct_tab_bytes(const srk_plan_s* p);
srk_status direct_build_tables(srk_plan_s* p, int kern, cudaStream_t s);
srk_status direct_forward(srk_plan_s* p, const void* E, const void* I, void* R, int B, cudaStream_t s);

// Tensor-core row pass of the FP16/BF16 forms at tile 512 (hybrid.cu).
bool tensor_rows_supported(const srk_plan_s* p, std::string* why);
size_t tensor_rows_tab_bytes(const srk_plan_s* p);
size_t tensor_rows_g_bytes(const srk_plan_s* p);
srk_status tensor_rows_build_tables(srk_plan_s* p, cudaStream_t s);
srk_status tensor_rows_p2(srk_plan_s* p, const __half* planes, const unsigned int* mx, int c, float2* scratch,
                          size_t per, size_t s1, int S, int P, cudaStream_t s);
size_t tensor_rows_p1g_tab_bytes();
srk_status tensor_rows_p1g_store_map(const __half* planes, int c, CUtensorMap* out);
srk_status tensor_rows_p1g_tables(srk_plan_s* p, cudaStream_t s);
srk_status tensor_rows_p1g_maps(const srk_plan_s* p, const void* img, int N, int nimg, CUtensorMap* tmap,
                                CUtensorMap* smap);
// Tensor map of a chunk's FP16 planes [2M][c][M] with the given box.
srk_status tensor_rows_plane_map(const __half* planes, int c, unsigned box_x, unsigned box_w, unsigned box_p,
                                 CUtensorMap* out, bool swizzle128 = false);

// Spectrum kernels defined in spectra.cuh (compiled once, in srk_abi.cu) and
// launched from the other translation units too.
__global__ void k_relayout(const float2* __restrict__ ref, int M, float scale, float2* __restrict__ full);
__global__ void k_fft_twiddles(float2* __restrict__ tw, int M);

}  // namespace srk
