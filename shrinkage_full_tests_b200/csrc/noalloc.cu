// noalloc.cu — the training forward for callers that cannot allocate device
// memory.
//
// Some callers may not call cudaMalloc at all: code that runs inside
// another framework's memory pool or under a strict memory budget, plug-ins
// loaded into a host that owns every device allocation, or code on a path
// that must not touch the allocator (an allocation there can synchronise the
// device or fail unpredictably).  srk_training_forward_noalloc serves them:
// the caller passes inputs, outputs and spectra, and every byte of scratch
// comes from one fixed array compiled into this library.
//
// The scratch array: kNoAllocScratchBytes (32 MiB) of device memory, a
// file-scope __device__ variable, so every GPU that loads the library holds
// it until the process exits.  It stores the FFT twiddle table, the
// re-laid-out kernel spectra (2 x M^2 complex) and a chunk of work tiles
// (image pairs); the batch is processed chunk by chunk.
//
// Set-up: the array's host-side name is only a stand-in; the device address
// comes from cudaGetSymbolAddress, resolved once per device (with that
// device current) by the first call on that device and cached.  Make that
// first call outside any CUDA stream capture.
//
// Sharing: all calls share the one array and it keeps the last call's
// contents.  Nothing in it needs to start at zero (each call writes every
// element it later reads), but two calls whose work overlaps on the GPU —
// different streams, or different host threads — race on it.  Serialise
// them (one stream, or events).
#include <mutex>

#include "internal.h"

using namespace srk;

namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device (resolved once
// per device).
srk_status noalloc_scratch(void** out) {
  int dev = 0;
  SRK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(SRK_ERR_UNSUPPORTED, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return SRK_OK;
}

}  // namespace

extern "C" srk_status srk_training_forward_noalloc(const float* d_E, const float* d_I, const void* d_Gx_freq,
                                                   const void* d_Gy_freq, int N, int W, int erosion, float dx, int B,
                                                   srk_stream_t stream, float* d_R) {
  g_last_error.clear();
  if (!d_E || !d_I || !d_Gx_freq || !d_Gy_freq || !d_R) return fail(SRK_ERR_INVALID_ARG, "NULL pointer");
  if (N < 3 || erosion < 0 || W != N - 2 * erosion || W < 1 || B < 1)
    return fail(SRK_ERR_INVALID_ARG, "need N>=3, erosion>=0, W == N-2*erosion >= 1, B >= 1 (N=%d W=%d erosion=%d B=%d)",
                N, W, erosion, B);
  if (!(dx > 0.f) || !std::isfinite(dx)) return fail(SRK_ERR_INVALID_ARG, "dx=%g must be positive", dx);
  // The spectra come at size N and are used as they are: the tile is the
  // whole image, so N must be one of the built tile sizes.
  if (N != 128 && N != 256 && N != 512)
    return fail(SRK_ERR_UNSUPPORTED, "no-alloc forward supports N in {128, 256, 512} (got %d)", N);
  const int M = N, S = M - 2 * erosion;
  if (S < 8) return fail(SRK_ERR_UNSUPPORTED, "erosion=%d leaves no valid outputs in a %d tile", erosion, M);
  // scratch layout: [twiddles M][Gx M*M][Gy M*M][work tiles ...]
  const size_t fixed = (size_t)M + 2 * (size_t)M * M;
  const size_t per_wt = (size_t)M * M + 2 * (size_t)M * s2_pitch(S);  // S1 + S2 of one forward work tile
  const size_t cap = kNoAllocScratchBytes / sizeof(float2);
  if (fixed + per_wt > cap)
    return fail(SRK_ERR_UNSUPPORTED, "N=%d needs %zu bytes of scratch for one work tile, the array holds %zu", N,
                (fixed + per_wt) * sizeof(float2), kNoAllocScratchBytes);
  void* base = nullptr;
  SRK_TRY(noalloc_scratch(&base));
  float2* sc = static_cast<float2*>(base);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

  // A plan view over the static array (host struct on the stack; nothing is allocated).
  srk_plan_s view;
  SRK_CUDA(cudaGetDevice(&view.device));
  SRK_CUDA(cudaDeviceGetAttribute(&view.nsm, cudaDevAttrMultiProcessorCount, view.device));
  view.N = N; view.W = W; view.e = erosion; view.dx = dx; view.B_max = B; view.spectra_M = N;
  view.dtype = SRK_F32;
  view.M = M; view.S = S; view.T = 1; view.Ta = 1;
  view.tw = sc;
  view.G[0] = sc + M;
  view.G[1] = sc + M + (size_t)M * M;
  view.have_G = true;
  view.scratch = sc + fixed;
  view.scratch_bytes = (cap - fixed) * sizeof(float2);
  view.schedule = SRK_SCHEDULE_THREE_PASS;

  // the twiddles and the spectrum re-layout of the plans (same kernels, so
  // the result equals srk_training_forward's with a plan at tile size N)
  k_fft_twiddles<<<(M + 127) / 128, 128, 0, s>>>(view.tw, M);
  const float scale = (dx * dx) / ((float)M * (float)M);
  k_relayout<<<dim3((M + 127) / 128, M), 128, 0, s>>>(static_cast<const float2*>(d_Gx_freq), M, scale, view.G[0]);
  k_relayout<<<dim3((M + 127) / 128, M), 128, 0, s>>>(static_cast<const float2*>(d_Gy_freq), M, scale, view.G[1]);
  SRK_CUDA(cudaGetLastError());

  OpArgs a;
  std::memset(&a, 0, sizeof(a));
  a.N = N; a.W = W; a.e = erosion;
  a.E = d_E; a.I = d_I; a.out0 = d_R;
  Geom g;
  std::memset(&g, 0, sizeof(g));
  g.M = M; g.e = erosion; g.S = S; g.T = 1; g.Nin = N; g.Wout = W; g.TT = 1; g.U = B;
  g.N = N; g.W = W;
  return launch_conv<OP_FWD, float>(&view, a, g, false, s);
}
