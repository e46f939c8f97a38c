// srk_abi.cu — host side of the C ABI declared in include/srk_b200.h:
// argument validation, plans (scratch, spectra, tile geometry), and the
// launch sequences of every operator.  No computation happens on the host;
// every path launches the kernels of engine.cuh / spectra.cuh and fails with
// a status if they cannot run.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <sys/stat.h>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "internal.h"
#include "spectra.cuh"

using namespace srk;

namespace {

// One NVTX range per operator call (visible in Nsight timelines; a no-op
// without a tool attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace



namespace {

// ---- tile choice -------------------------------------------------------------
// FFT work per image ~ T^2 * M^2 * log2(M) for the forward geometry; choose
// the cheapest M whose valid stride S = M - 2e keeps at least 16 outputs.
int choose_tile(int N, int W, int e) {
  const int cand[3] = {128, 256, 512};
  int best = 0;
  double best_cost = 0;
  for (int M : cand) {
    const int S = M - 2 * e;
    if (S < 16) continue;
    const int T = (W + S - 1) / S;
    const double lg = std::log2((double)M);
    const double cost = (double)T * T * M * M * lg;
    if (best == 0 || cost < best_cost * 0.98) { best = M; best_cost = cost; }
  }
  return best;
}

Geom fwd_geom(const srk_plan_s* p, int B) {
  Geom g;
  std::memset(&g, 0, sizeof(g));
  g.M = p->M; g.e = p->e; g.S = p->S; g.T = p->T;
  g.Nin = p->N; g.Wout = p->W; g.TT = p->T * p->T; g.U = B * g.TT;
  g.N = p->N; g.W = p->W; g.wout_n = 0;
  return g;
}
Geom adj_geom(const srk_plan_s* p, int B) {
  Geom g;
  std::memset(&g, 0, sizeof(g));
  g.M = p->M; g.e = p->e; g.S = p->S; g.T = p->Ta;
  g.Nin = p->N + 2 * p->e; g.Wout = p->N; g.TT = p->Ta * p->Ta; g.U = B * g.TT;
  g.N = p->N; g.W = p->W; g.wout_n = 1;
  return g;
}

size_t wt_bytes(int M, int S) {
  const size_t P = (size_t)s2_pitch(S);
  const size_t fwd = (size_t)M * M + 2 * P * M;
  const size_t adj = 2 * (size_t)M * M + P * M;
  return sizeof(float2) * (fwd > adj ? fwd : adj);
}

// ---- launch helpers -------------------------------------------------------------
// Element type of the plan's image buffers.
template <int OP>
srk_status launch_conv_dt(srk_plan_s* p, const OpArgs& a, const Geom& g, bool conjG, cudaStream_t s) {
  switch (p->dtype) {
    case SRK_F32: return launch_conv<OP, float>(p, a, g, conjG, s);
    case SRK_F16: return launch_conv<OP, __half>(p, a, g, conjG, s);
    case SRK_BF16: return launch_conv<OP, __nv_bfloat16>(p, a, g, conjG, s);
  }
  return fail(SRK_ERR_UNSUPPORTED, "dtype %d", (int)p->dtype);
}

// The W-sized intermediate of the VJP and the tangent-adjoint (wx, wy = u*v
// between the engine's P3 and the transposed stencil) lives in a buffer the
// plan allocates at creation (2 W^2 B_max floats): no operator allocates.
srk_status ensure_wbuf(srk_plan_s* p, size_t bytes, cudaStream_t) {
  if (p->wbuf_bytes >= bytes) return SRK_OK;
  return fail(SRK_ERR_UNSUPPORTED,
              "the call needs %zu bytes of derivative intermediate, the plan holds %zu (2 W^2 B_max floats)", bytes,
              p->wbuf_bytes);
}

template <typename T>
void adj_wrt_f_t(srk_plan_s* p, const float* wx, const float* wy, const void* v, const void* ux, const void* uy, int B,
                 void* out, cudaStream_t s) {
  const dim3 blk(32, 8);
  const dim3 grd((p->N + 31) / 32, (p->N + 8 * kStencilCols - 1) / (8 * kStencilCols), B);
  if (ux)
    k_adj_wrt_f<T, true><<<grd, blk, 0, s>>>(nullptr, nullptr, static_cast<const T*>(v), static_cast<const T*>(ux),
                                             static_cast<const T*>(uy), p->N, p->W, p->e, B, static_cast<T*>(out));
  else
    k_adj_wrt_f<T, false><<<grd, blk, 0, s>>>(wx, wy, nullptr, nullptr, nullptr, p->N, p->W, p->e, B,
                                              static_cast<T*>(out));
}

srk_status adj_wrt_f(srk_plan_s* p, const float* wx, const float* wy, const void* v, const void* ux,
                     const void* uy, int B, void* out, cudaStream_t s) {
  switch (p->dtype) {
    case SRK_F32: adj_wrt_f_t<float>(p, wx, wy, v, ux, uy, B, out, s); break;
    case SRK_F16: adj_wrt_f_t<__half>(p, wx, wy, v, ux, uy, B, out, s); break;
    case SRK_BF16: adj_wrt_f_t<__nv_bfloat16>(p, wx, wy, v, ux, uy, B, out, s); break;
  }
  return cuda_status(cudaGetLastError(), "adj_wrt_f launch");
}

// ---- spectra -----------------------------------------------------------------------
// FP64 twiddle table (cos, sin)(2 pi m / M) built on the device.
srk_status build_tab64(double2* tab, int M, cudaStream_t s) {
  k_twiddles64<<<(M + 127) / 128, 128, 0, s>>>(tab, M);
  return cuda_status(cudaGetLastError(), "twiddle table launch");
}

// Spatial kernel (double, column-major KW x KW) -> engine spectrum at size M.
// tab: FP64 twiddles at size M; P: KW x M double2 of workspace.
srk_status spectrum_from_spatial(const double* Kd, int KW, int M, const double2* tab, double2* P, double scale,
                                 float2* full, float2* ref, cudaStream_t s) {
  k_dft_cols<<<dim3((M + 127) / 128, KW), 128, 0, s>>>(Kd, KW, M, tab, P);
  k_dft_rows<<<dim3((M + 127) / 128, M), 128, 0, s>>>(P, KW, M, tab, scale, full, ref);
  return cuda_status(cudaGetLastError(), "kernel DFT launch");
}

// Caller spectrum (reference layout, size spectra_M) -> the plan's engine
// layout at the tile size, and the kernel in space (kd[k], FP64, on its
// (2e+1)^2 support) for the direct schedule.  Stream-ordered; uses only the
// plan's import workspace (no allocation, no host synchronisation), so it
// may run under stream capture.
srk_status import_one(srk_plan_s* p, int k, const float2* ref, float2* full, cudaStream_t s) {
  const int Mr = p->spectra_M;
  // dx^2 / M^2 folded into the spectrum (srkConvOaS applies dx*dx/(M*M), srk_forward.cuh:380)
  const float scale = (p->dx * p->dx) / ((float)p->M * (float)p->M);
  const int c = p->e;
  const int KW = 2 * c + 1;
  // spatial recovery on the kernel support, in FP64
  k_recover_a<<<dim3((KW + 127) / 128, Mr / 2 + 1), 128, 0, s>>>(ref, Mr, c, p->imp_tabr, p->imp_Tm);
  k_recover_b<<<(KW * KW + 127) / 128, 128, 0, s>>>(p->imp_Tm, Mr, c, p->imp_tabr, p->kd[k]);
  SRK_CUDA(cudaGetLastError());
  if (Mr == p->M) {
    // same FFT size: the caller's values as they are
    k_relayout<<<dim3((Mr + 127) / 128, Mr), 128, 0, s>>>(ref, Mr, scale, full);
    return cuda_status(cudaGetLastError(), "relayout");
  }
  // different FFT size: the spectrum of the recovered kernel at the tile size
  return spectrum_from_spatial(p->kd[k], KW, p->M, p->imp_tab, p->imp_P, (double)scale, full, nullptr, s);
}

// Band tables of the tensor-core schedules from the bound kernel (when one
// of them is selected).
srk_status refresh_direct(srk_plan_s* p, cudaStream_t s) {
  p->direct_ready = false;
  p->hyb_ready = false;
  if (!p->have_G) return SRK_OK;
  if (p->schedule == SRK_SCHEDULE_DIRECT) {
    SRK_TRY(direct_build_tables(p, 0, s));
    SRK_TRY(direct_build_tables(p, 1, s));
    p->direct_ready = true;
  } else if (p->schedule == SRK_SCHEDULE_TENSOR_ROWS) {
    SRK_TRY(tensor_rows_build_tables(p, s));
    p->hyb_ready = true;
  }
  return SRK_OK;
}

srk_status import_spectra(srk_plan_s* p, const void* gx, const void* gy, cudaStream_t s) {
  if (!gx || !gy) return fail(SRK_ERR_INVALID_ARG, "kernel spectra are NULL");
  SRK_TRY(import_one(p, 0, static_cast<const float2*>(gx), p->G[0], s));
  SRK_TRY(import_one(p, 1, static_cast<const float2*>(gy), p->G[1], s));
  p->src[0] = gx;
  p->src[1] = gy;
  p->have_G = true;
  return refresh_direct(p, s);
}

srk_status bind_spectra(srk_plan_s* p, const void* gx, const void* gy, cudaStream_t s) {
  if (gx == nullptr && gy == nullptr) {
    if (!p->have_G) return fail(SRK_ERR_INVALID_ARG, "no kernel spectra given and none set on the plan");
    return SRK_OK;
  }
  if (p->have_G && gx == p->src[0] && gy == p->src[1]) return SRK_OK;
  return import_spectra(p, gx, gy, s);
}

srk_status check_dims(const srk_plan_s* p, int N, int W, int e, float dx) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  if (N != p->N || W != p->W || e != p->e)
    return fail(SRK_ERR_INVALID_ARG, "sizes (N=%d W=%d erosion=%d) differ from the plan (N=%d W=%d erosion=%d)", N,
                W, e, p->N, p->W, p->e);
  if (dx != p->dx) return fail(SRK_ERR_INVALID_ARG, "dx=%g differs from the plan's dx=%g", dx, p->dx);
  return SRK_OK;
}

srk_status check_batch(const srk_plan_s* p, int B) {
  if (B < 1 || B > p->B_max) return fail(SRK_ERR_INVALID_ARG, "B=%d outside [1, B_max=%d]", B, p->B_max);
  return SRK_OK;
}

#define SRK_NONNULL(ptr) \
  do { if (!(ptr)) return fail(SRK_ERR_INVALID_ARG, "%s is NULL", #ptr); } while (0)

OpArgs base_args(const srk_plan_s* p) {
  OpArgs a;
  std::memset(&a, 0, sizeof(a));
  a.N = p->N;
  a.W = p->W;
  a.e = p->e;
  return a;
}

srk_status set_device(const srk_plan_s* p) { return cuda_status(cudaSetDevice(p->device), "cudaSetDevice"); }

// Report (once) a bounded wait that gave up in an already completed
// persistent launch of this plan.
srk_status check_mailbox(srk_plan_s* p) {
  if (!p->mailbox_pending) return SRK_OK;
  const cudaError_t q = cudaEventQuery(p->mailbox_ev);
  if (q == cudaErrorNotReady) return SRK_OK;
  if (q != cudaSuccess) return cuda_status(q, "mailbox event");
  p->mailbox_pending = false;
  if (p->mailbox[0]) {
    const unsigned int where = p->mailbox[1];
    p->mailbox[0] = 0;
    return fail(SRK_ERR_TIMEOUT, "a bounded device-side wait gave up (site %u); that call's outputs are incomplete",
                where);
  }
  return SRK_OK;
}

srk_status enter(srk_plan_s* p, cudaStream_t s) {
  SRK_TRY(set_device(p));
  if (stream_capturing(s)) return SRK_OK;
  return check_mailbox(p);
}

// dL/dg through the adjoint engine: h = v*df (+ dv*f' for the tangent-adjoint)
srk_status run_adj_g(srk_plan_s* p, const void* v, const void* dv, const void* f, const void* df, int B,
                     bool conj, void* out, cudaStream_t s) {
  OpArgs a = base_args(p);
  a.v = v; a.dv = dv; a.I = f; a.dI = df; a.out0 = out;
  return launch_conv_dt<OP_ADJ>(p, a, adj_geom(p, B), conj, s);
}

// ---- autotuner ------------------------------------------------------------------
// Times every (tile size, schedule) candidate of the forward operator on
// synthetic device data and remembers the fastest per device and
// configuration in a small text cache (one "key value" line per entry).
__global__ void k_fill_pattern(float* __restrict__ x, size_t n, unsigned seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned h = (unsigned)i * 2654435761u ^ seed;
    h ^= h >> 15; h *= 2246822519u; h ^= h >> 13;
    x[i] = (float)(h & 0xffffff) * (1.0f / 16777216.0f);
  }
}

std::string tune_cache_path() {
  const char* env = getenv("SRK_TUNE_CACHE");
  if (env && *env) return env;
  const char* home = getenv("HOME");
  return std::string(home ? home : "/tmp") + "/.cache/srk_b200_tune.txt";
}

std::string tune_key(int N, int W, int e, int B, srk_dtype dt) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  std::string name(prop.name);
  for (auto& c : name) if (c == ' ') c = '_';
  int bb = 1;
  while (bb < B) bb <<= 1;  // batch bucket
  char buf[256];
  snprintf(buf, sizeof(buf), "%s:N%d:W%d:e%d:B%d:t%d", name.c_str(), N, W, e, bb, (int)dt);
  return buf;
}

bool tune_lookup(const std::string& key, int* M, int* sched) {
  FILE* f = fopen(tune_cache_path().c_str(), "r");
  if (!f) return false;
  char k[256];
  int m = 0, sc = 0;
  bool found = false;
  // entries are appended one line per write (ranks of one node may share
  // the file); anything that is not a valid (tile, schedule) pair is ignored
  while (fscanf(f, "%255s %d %d", k, &m, &sc) == 3)
    if (key == k && (m == 128 || m == 256 || m == 512) && (sc == 0 || sc == 1)) {
      *M = m;
      *sched = sc;
      found = true;
    }
  fclose(f);
  return found;
}

void tune_store(const std::string& key, int M, int sched) {
  const std::string path = tune_cache_path();
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) mkdir(path.substr(0, slash).c_str(), 0755);  // best effort
  FILE* f = fopen(path.c_str(), "a");
  if (!f) return;
  fprintf(f, "%s %d %d\n", key.c_str(), M, sched);
  fclose(f);
}

}  // namespace

// ============================== C ABI ========================================
extern "C" {

int srk_version(void) { return 100; }

const char* srk_status_string(srk_status s) {
  switch (s) {
    case SRK_OK: return "SRK_OK";
    case SRK_ERR_INVALID_ARG: return "SRK_ERR_INVALID_ARG";
    case SRK_ERR_UNSUPPORTED: return "SRK_ERR_UNSUPPORTED";
    case SRK_ERR_ALLOC: return "SRK_ERR_ALLOC";
    case SRK_ERR_TIMEOUT: return "SRK_ERR_TIMEOUT";
    case SRK_ERR_CUDA: return "SRK_ERR_CUDA";
  }
  return "SRK_ERR_UNKNOWN";
}

const char* srk_last_error(void) { return g_last_error.c_str(); }

srk_status srk_plan_create(srk_plan* out, int N, int W, int erosion, float dx, int B_max, int spectra_M,
                           srk_dtype dtype, int tile_M, size_t budget) {
  g_last_error.clear();
  if (!out) return fail(SRK_ERR_INVALID_ARG, "plan out-pointer is NULL");
  *out = nullptr;
  if (N < 3 || erosion < 0 || W != N - 2 * erosion || W < 1)
    return fail(SRK_ERR_INVALID_ARG, "need N>=3, erosion>=0, W == N-2*erosion >= 1 (got N=%d W=%d erosion=%d)", N, W,
                erosion);
  if (B_max < 1) return fail(SRK_ERR_INVALID_ARG, "B_max=%d < 1", B_max);
  if (spectra_M < 2 || (spectra_M & 1)) return fail(SRK_ERR_INVALID_ARG, "spectra_M=%d must be even", spectra_M);
  if (spectra_M < 2 * erosion + 1)
    return fail(SRK_ERR_INVALID_ARG, "spectra_M=%d smaller than the kernel support 2*erosion+1", spectra_M);
  if (dtype != SRK_F32 && dtype != SRK_F16 && dtype != SRK_BF16) return fail(SRK_ERR_INVALID_ARG, "bad dtype %d", (int)dtype);
  if (!(dx > 0.f) || !std::isfinite(dx)) return fail(SRK_ERR_INVALID_ARG, "dx=%g must be positive", dx);
  int M = tile_M;
  int sched = SRK_SCHEDULE_THREE_PASS;
  if (M == SRK_TILE_AUTOTUNE) {
    const srk_status st = srk_autotune(N, W, erosion, dx, B_max, dtype, &M, &sched);
    if (st != SRK_OK) return st;
  }
  if (M == 0) M = choose_tile(N, W, erosion);
  if (M == 0)
    return fail(SRK_ERR_UNSUPPORTED, "erosion=%d too large for the 512 tile (needs stride >= 16)", erosion);
  if (!(M == 128 || M == 256 || M == 512)) return fail(SRK_ERR_INVALID_ARG, "tile_M=%d not in {128,256,512}", M);
  if (M - 2 * erosion < 8) return fail(SRK_ERR_UNSUPPORTED, "tile_M=%d leaves no valid stride for erosion=%d", M, erosion);

  srk_plan_s* p = new srk_plan_s();
  cudaGetDevice(&p->device);
  cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, p->device);
  p->N = N; p->W = W; p->e = erosion; p->dx = dx; p->B_max = B_max; p->spectra_M = spectra_M; p->dtype = dtype;
  p->M = M; p->S = M - 2 * erosion;
  p->schedule = sched;
  p->T = (W + p->S - 1) / p->S;
  p->Ta = (N + p->S - 1) / p->S;
  const size_t nwt_max = std::max<size_t>({(size_t)(B_max * (size_t)p->T * p->T + 1) / 2,
                                           (size_t)B_max * p->T * p->T,
                                           (size_t)(B_max * (size_t)p->Ta * p->Ta + 1) / 2});
  const size_t per = wt_bytes(M, p->S);
  // default scratch: 8 GiB, at most 1/16 of the device memory, at least
  // 256 MiB.  At B=5000 on the B200 it holds the whole N=256 batch (one
  // chunk: -4% against 1 GiB) and N=512 runs in 15 launches (-1.3%); the
  // ring of chunks keeps smaller budgets within a few percent of it.
  size_t cap = budget;
  if (!cap) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    cap = std::max<size_t>((size_t)256 << 20, std::min<size_t>((size_t)8 << 30, total_b / 16));
  }
  size_t chunk = cap / per;
  if (chunk < 1) chunk = 1;
  if (chunk > nwt_max) chunk = nwt_max;
  if (chunk > 65535) chunk = 65535;
  p->chunk = (int)chunk;
  p->scratch_bytes = per * chunk;

  auto cleanup = [&](srk_status st) { srk_plan_destroy(p); return st; };
  cudaError_t err;
  if ((err = cudaMalloc(reinterpret_cast<void**>(&p->scratch), p->scratch_bytes)) != cudaSuccess)
    return cleanup(cuda_status(err, "scratch allocation"));
  for (int i = 0; i < 2; ++i)
    if ((err = cudaMalloc(reinterpret_cast<void**>(&p->G[i]), sizeof(float2) * (size_t)M * M)) != cudaSuccess)
      return cleanup(cuda_status(err, "spectrum allocation"));
  if ((err = cudaMalloc(reinterpret_cast<void**>(&p->tw), sizeof(float2) * M)) != cudaSuccess)
    return cleanup(cuda_status(err, "twiddle allocation"));
  // the derivative operators' intermediate (ensure_wbuf), allocated here once
  p->wbuf_bytes = 2 * (size_t)W * W * (size_t)B_max * sizeof(float);
  if ((err = cudaMalloc(reinterpret_cast<void**>(&p->wbuf), p->wbuf_bytes)) != cudaSuccess) {
    p->wbuf_bytes = 0;
    return cleanup(cuda_status(err, "derivative intermediate allocation"));
  }
  if ((err = cudaMalloc(reinterpret_cast<void**>(&p->ctl), sizeof(Ctl))) != cudaSuccess)
    return cleanup(cuda_status(err, "control block allocation"));
  if ((err = cudaHostAlloc(reinterpret_cast<void**>(&p->mailbox), 2 * sizeof(unsigned int), cudaHostAllocDefault)) !=
      cudaSuccess)
    return cleanup(cuda_status(err, "mailbox allocation"));
  p->mailbox[0] = p->mailbox[1] = 0;
  if ((err = cudaHostAlloc(reinterpret_cast<void**>(&p->mailbox_spins), sizeof(unsigned long long),
                           cudaHostAllocDefault)) != cudaSuccess)
    return cleanup(cuda_status(err, "mailbox allocation"));
  *p->mailbox_spins = 0;
  if ((err = cudaEventCreateWithFlags(&p->mailbox_ev, cudaEventDisableTiming)) != cudaSuccess)
    return cleanup(cuda_status(err, "event creation"));
  for (cudaStream_t* st : {&p->ps1, &p->ps3})
    if ((err = cudaStreamCreateWithFlags(st, cudaStreamNonBlocking)) != cudaSuccess)
      return cleanup(cuda_status(err, "stream creation"));
  if ((err = cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming)) != cudaSuccess)
    return cleanup(cuda_status(err, "event creation"));
  for (int r = 0; r < srk_plan_s::kRing; ++r)
    for (cudaEvent_t* ev : {&p->ev1[r], &p->ev2[r], &p->ev3[r]})
      if ((err = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess)
        return cleanup(cuda_status(err, "event creation"));
  // spectrum import workspace (sizes in internal.h)
  {
    const size_t KW = 2 * (size_t)erosion + 1;
    const size_t Mr = (size_t)spectra_M;
    struct { void** ptr; size_t bytes; } bufs[] = {
        {reinterpret_cast<void**>(&p->imp_tab), sizeof(double2) * (size_t)M},
        {reinterpret_cast<void**>(&p->imp_tabr), sizeof(double2) * Mr},
        {reinterpret_cast<void**>(&p->imp_P), sizeof(double2) * KW * (size_t)M},
        {reinterpret_cast<void**>(&p->imp_Tm), sizeof(double2) * (Mr / 2 + 1) * KW},
        {reinterpret_cast<void**>(&p->imp_Kd), sizeof(double) * KW * KW},
        {reinterpret_cast<void**>(&p->kd[0]), sizeof(double) * KW * KW},
        {reinterpret_cast<void**>(&p->kd[1]), sizeof(double) * KW * KW},
        {reinterpret_cast<void**>(&p->direct_err), 4 * sizeof(unsigned int)}};
    for (auto& b : bufs)
      if ((err = cudaMalloc(b.ptr, b.bytes)) != cudaSuccess) return cleanup(cuda_status(err, "import workspace"));
  }
  // twiddle tables built on the device: the engine's per-pass float blocks
  // (k_fft_twiddles, shared with the no-allocation forward) and the FP64
  // tables of the spectrum import
  k_fft_twiddles<<<(M + 127) / 128, 128>>>(p->tw, M);
  k_twiddles64<<<(M + 127) / 128, 128>>>(p->imp_tab, M);
  k_twiddles64<<<(spectra_M + 127) / 128, 128>>>(p->imp_tabr, spectra_M);
  if ((err = cudaMemset(p->direct_err, 0, 4 * sizeof(unsigned int))) != cudaSuccess)
    return cleanup(cuda_status(err, "error word"));
  if ((err = cudaGetLastError()) != cudaSuccess) return cleanup(cuda_status(err, "twiddle tables"));
  if ((err = cudaStreamSynchronize(0)) != cudaSuccess) return cleanup(cuda_status(err, "twiddle tables"));
  if (sched == SRK_SCHEDULE_DIRECT || sched == SRK_SCHEDULE_TENSOR_ROWS) {
    // the tuner chose a tensor-core schedule for the forward
    const srk_status st = srk_plan_set_schedule(p, (srk_schedule)sched);
    if (st != SRK_OK) return cleanup(st);
  }
  *out = p;
  return SRK_OK;
}

srk_status srk_plan_destroy(srk_plan p) {
  if (!p) return SRK_OK;
  cudaSetDevice(p->device);
  // work queued on any of the caller's streams may still use the plan's
  // buffers (cudaFree would synchronise the device as well)
  cudaDeviceSynchronize();
  if (p->scratch) cudaFree(p->scratch);
  if (p->G[0]) cudaFree(p->G[0]);
  if (p->G[1]) cudaFree(p->G[1]);
  if (p->tw) cudaFree(p->tw);
  for (void* q : {(void*)p->imp_tab, (void*)p->imp_tabr, (void*)p->imp_P, (void*)p->imp_Tm, (void*)p->imp_Kd,
                  (void*)p->kd[0], (void*)p->kd[1], (void*)p->direct_tabs, (void*)p->direct_err,
                  (void*)p->hyb_s1, (void*)p->hyb_tabs, (void*)p->hyb_g, (void*)p->hyb_mx, p->p1g_tab})
    if (q) cudaFree(q);
  if (p->wbuf) cudaFree(p->wbuf);
  for (auto& kv : p->tables) {
    if (kv.second.tiles) cudaFree(kv.second.tiles);
    if (kv.second.imgs) cudaFree(kv.second.imgs);
  }
  if (p->ctl) cudaFree(p->ctl);
  if (p->mailbox) cudaFreeHost(p->mailbox);
  if (p->mailbox_spins) cudaFreeHost(p->mailbox_spins);
  if (p->mailbox_ev) cudaEventDestroy(p->mailbox_ev);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  for (int r = 0; r < srk_plan_s::kRing; ++r)
    for (cudaEvent_t ev : {p->ev1[r], p->ev2[r], p->ev3[r]})
      if (ev) cudaEventDestroy(ev);
  for (cudaStream_t st : {p->ps1, p->ps3})
    if (st) cudaStreamDestroy(st);
  delete p;
  return SRK_OK;
}

srk_status srk_plan_get_info(srk_plan p, srk_plan_info* info) {
  if (!p || !info) return fail(SRK_ERR_INVALID_ARG, "NULL plan or info");
  info->N = p->N; info->W = p->W; info->erosion = p->e; info->B_max = p->B_max; info->spectra_M = p->spectra_M;
  info->dx = p->dx; info->tile_M = p->M; info->tile_stride = p->S; info->tiles = p->T; info->tiles_adj = p->Ta;
  info->chunk_wt = p->chunk; info->scratch_bytes = p->scratch_bytes; info->dtype = p->dtype;
  info->schedule = p->schedule; info->last_launches = p->last_launches; info->last_grid = p->last_grid;
  info->last_lag = p->last_lag; info->last_nslot = p->last_nslot;
  info->last_spins = p->mailbox_spins ? *p->mailbox_spins : 0;
  return SRK_OK;
}

srk_status srk_plan_set_schedule(srk_plan p, srk_schedule sch) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  if (sch != SRK_SCHEDULE_PERSISTENT && sch != SRK_SCHEDULE_THREE_PASS && sch != SRK_SCHEDULE_DIRECT &&
      sch != SRK_SCHEDULE_TENSOR_ROWS)
    return fail(SRK_ERR_INVALID_ARG, "bad schedule %d", (int)sch);
  if (sch == SRK_SCHEDULE_TENSOR_ROWS) {
    std::string why;
    if (!tensor_rows_supported(p, &why)) return fail(SRK_ERR_UNSUPPORTED, "tensor-row schedule: %s", why.c_str());
    SRK_TRY(set_device(p));
    SRK_CUDA(cudaDeviceSynchronize());  // the bound spectra may still be in flight on the caller's stream
    if (!p->hyb_tabs) SRK_CUDA(cudaMalloc(reinterpret_cast<void**>(&p->hyb_tabs), tensor_rows_tab_bytes(p)));
    if (!p->hyb_g) SRK_CUDA(cudaMalloc(reinterpret_cast<void**>(&p->hyb_g), tensor_rows_g_bytes(p)));
    if (!p->hyb_s1) {
      // FP16 column spectra: 2 parts x M x M halves per work tile the scratch holds
      const size_t bytes = (size_t)p->chunk * 2 * p->M * p->M * sizeof(__half);
      SRK_CUDA(cudaMalloc(reinterpret_cast<void**>(&p->hyb_s1), bytes));
      p->hyb_s1_bytes = bytes;
    }
    if (!p->hyb_mx) SRK_CUDA(cudaMalloc(reinterpret_cast<void**>(&p->hyb_mx), (size_t)p->chunk * sizeof(unsigned int)));
    if (!p->p1g_tab) {
      SRK_CUDA(cudaMalloc(&p->p1g_tab, tensor_rows_p1g_tab_bytes()));
      SRK_TRY(tensor_rows_p1g_tables(p, nullptr));
    }
    p->schedule = sch;
    SRK_TRY(refresh_direct(p, nullptr));
    SRK_CUDA(cudaStreamSynchronize(nullptr));
    return SRK_OK;
  }
  if (sch == SRK_SCHEDULE_DIRECT) {
    std::string why;
    if (!direct_supported(p, p->N, &why)) return fail(SRK_ERR_UNSUPPORTED, "direct schedule: %s", why.c_str());
    SRK_TRY(set_device(p));
    SRK_CUDA(cudaDeviceSynchronize());  // the bound kernel (kd) may still be in flight on the caller's stream
    if (!p->direct_tabs) SRK_CUDA(cudaMalloc(reinterpret_cast<void**>(&p->direct_tabs), direct_tab_bytes(p)));
    p->schedule = sch;
    // band tables of an already bound kernel (legacy stream, then ready)
    SRK_TRY(refresh_direct(p, nullptr));
    SRK_CUDA(cudaStreamSynchronize(nullptr));
    return SRK_OK;
  }
  p->schedule = sch;
  p->direct_ready = false;
  p->hyb_ready = false;
  return SRK_OK;
}

srk_status srk_plan_set_persistent(srk_plan p, int lag, int grid, int prefetch) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  if (lag < 0 || lag > kMaxSlots / 2 - 1 || grid < 0 || (prefetch != 0 && prefetch != 1))
    return fail(SRK_ERR_INVALID_ARG, "bad persistent parameters lag=%d grid=%d prefetch=%d", lag, grid, prefetch);
  p->persist_lag = lag;
  p->persist_grid = grid;
  p->persist_prefetch = prefetch;
  return SRK_OK;
}

srk_status srk_plan_sync(srk_plan p, srk_stream_t s) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_TRY(set_device(p));
  SRK_CUDA(cudaStreamSynchronize(s));
  if (p->direct_err) {
    unsigned int derr = 0;
    SRK_CUDA(cudaMemcpy(&derr, p->direct_err, sizeof(derr), cudaMemcpyDeviceToHost));
    if (derr) {
      SRK_CUDA(cudaMemset(p->direct_err, 0, sizeof(derr)));
      return fail(SRK_ERR_TIMEOUT,
                  "a tensor-core schedule stopped early (site %u: 1-13 a bounded wait gave up, 14-15 a shared "
                  "memory block off its alignment); outputs incomplete",
                  derr);
    }
  }
  if (p->graph_mailbox && p->mailbox[0]) {
    // written by a persistent launch replayed from a captured graph
    const unsigned int where = p->mailbox[1];
    p->mailbox[0] = 0;
    p->mailbox_pending = false;
    return fail(SRK_ERR_TIMEOUT, "a bounded device-side wait gave up (site %u); that call's outputs are incomplete",
                where);
  }
  return check_mailbox(p);
}

srk_status srk_debug_wait_selftest(srk_plan p, unsigned long long spin_limit, srk_stream_t s) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  if (spin_limit == 0 || spin_limit > (1ull << 26)) return fail(SRK_ERR_INVALID_ARG, "spin_limit out of range");
  SRK_TRY(enter(p, s));
  SRK_CUDA(cudaMemsetAsync(p->ctl, 0, sizeof(Ctl), s));
  k_wait_selftest<<<1, 32, 0, s>>>(p->ctl, spin_limit);
  SRK_CUDA(cudaGetLastError());
  SRK_CUDA(cudaMemcpyAsync(p->mailbox, &p->ctl->abort, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  SRK_CUDA(cudaEventRecord(p->mailbox_ev, s));
  p->mailbox_pending = true;
  return srk_plan_sync(p, s);
}

srk_status srk_plan_set_adj_convention(srk_plan p, srk_adj_convention c) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  if (c != SRK_ADJ_REFERENCE && c != SRK_ADJ_TRUE) return fail(SRK_ERR_INVALID_ARG, "bad convention %d", (int)c);
  p->conv = c;
  return SRK_OK;
}

srk_status srk_plan_import_spectra(srk_plan p, const void* gx, const void* gy, srk_stream_t stream) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_TRY(set_device(p));
  return import_spectra(p, gx, gy, stream);
}

srk_status srk_plan_set_kernel(srk_plan p, const float* Kx, const float* Ky, int KW, srk_stream_t s) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_NONNULL(Kx);
  SRK_NONNULL(Ky);
  if (KW < 1 || !(KW & 1) || KW > 2 * p->e + 1)
    return fail(SRK_ERR_INVALID_ARG, "KW=%d must be odd and <= 2*erosion+1=%d", KW, 2 * p->e + 1);
  SRK_TRY(set_device(p));
  const double scale = (double)p->dx * (double)p->dx / ((double)p->M * (double)p->M);
  const float* K[2] = {Kx, Ky};
  const int KWp = 2 * p->e + 1;
  for (int i = 0; i < 2; ++i) {
    // the kernel centred on the plan's full (2e+1)^2 support
    k_pad_centre<<<(KWp * KWp + 255) / 256, 256, 0, s>>>(K[i], KW, KWp, p->kd[i]);
    SRK_TRY(spectrum_from_spatial(p->kd[i], KWp, p->M, p->imp_tab, p->imp_P, scale, p->G[i], nullptr, s));
  }
  p->src[0] = p->src[1] = nullptr;
  p->have_G = true;
  return refresh_direct(p, s);
}

srk_status srk_green_tensor(float* Kx, float* Ky, int KW, double gamma, double R_w, double dx, srk_stream_t s) {
  SRK_NONNULL(Kx);
  SRK_NONNULL(Ky);
  if (KW < 1 || !(KW & 1)) return fail(SRK_ERR_INVALID_ARG, "KW=%d must be odd", KW);
  if (!(gamma > 0) || !(R_w > 0) || !(dx > 0)) return fail(SRK_ERR_INVALID_ARG, "gamma, R_w, dx must be > 0");
  k_green_tensor<<<(KW * KW + 127) / 128, 128, 0, s>>>(KW, gamma, R_w, dx, Kx, Ky);
  return cuda_status(cudaGetLastError(), "green tensor launch");
}

srk_status srk_precompute_kernel_freq(const float* K, int KW, int M, void* freq, srk_stream_t s) {
  SRK_NONNULL(K);
  SRK_NONNULL(freq);
  if (KW < 1 || !(KW & 1) || M < KW || (M & 1))
    return fail(SRK_ERR_INVALID_ARG, "need odd KW <= M, even M (KW=%d M=%d)", KW, M);
  // stream-ordered temporaries (no host synchronisation): FP64 kernel,
  // twiddle table and the column pass of the DFT
  double* Kd = nullptr;
  double2* tab = nullptr;
  double2* P = nullptr;
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&Kd), sizeof(double) * KW * KW, s));
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&tab), sizeof(double2) * (size_t)M, s));
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&P), sizeof(double2) * (size_t)KW * M, s));
  k_float_to_double<<<(KW * KW + 255) / 256, 256, 0, s>>>(K, Kd, KW * KW);
  SRK_TRY(build_tab64(tab, M, s));
  SRK_TRY(spectrum_from_spatial(Kd, KW, M, tab, P, 1.0, nullptr, static_cast<float2*>(freq), s));
  SRK_CUDA(cudaFreeAsync(P, s));
  SRK_CUDA(cudaFreeAsync(tab, s));
  SRK_CUDA(cudaFreeAsync(Kd, s));
  return SRK_OK;
}

// ---- typed operator bodies (element type = plan dtype) --------------------------
}  // extern "C"
namespace {

srk_status op_training_forward(const void* E, const void* I, const void* gx, const void* gy, int N, int W,
                               int erosion, float dx, int B, srk_stream_t s, void* R, srk_plan p) {
  const NvtxRange nvtx_range("srk_training_forward");
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_TRY(check_batch(p, B));
  SRK_NONNULL(E);
  SRK_NONNULL(I);
  SRK_NONNULL(R);
  if (p->spectra_M != N && (gx || gy))
    return fail(SRK_ERR_INVALID_ARG, "training spectra must be at size N=%d (plan has spectra_M=%d)", N, p->spectra_M);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  if (p->schedule == SRK_SCHEDULE_DIRECT) return direct_forward(p, E, I, R, B, s);
  OpArgs a = base_args(p);
  a.E = E; a.I = I; a.out0 = R;
  return launch_conv_dt<OP_FWD>(p, a, fwd_geom(p, B), false, s);
}

srk_status op_forward_oas(const void* E, const void* I, const void* gx, const void* gy, int N, int W, int erosion,
                          float dx, srk_stream_t s, void* R, srk_plan p, void* ux, void* uy) {
  const NvtxRange nvtx_range("srk_forward_oas");
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_NONNULL(E);
  SRK_NONNULL(I);
  SRK_NONNULL(R);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  OpArgs a = base_args(p);
  a.E = E; a.I = I; a.out0 = R; a.out_ux = ux; a.out_uy = uy;
  return launch_conv_dt<OP_FWD>(p, a, fwd_geom(p, 1), false, s);
}

srk_status op_adjoint(const void* v, const void* ux, const void* uy, const void* I, const void* gx, const void* gy,
                      int N, int W, int erosion, float dx, srk_stream_t s, void* dLdI, void* dLdE, srk_plan p) {
  const NvtxRange nvtx_range("srk_adjoint");
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_NONNULL(v);
  SRK_NONNULL(ux);
  SRK_NONNULL(uy);
  SRK_NONNULL(I);
  SRK_NONNULL(dLdI);
  SRK_NONNULL(dLdE);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(adj_wrt_f(p, nullptr, nullptr, v, ux, uy, 1, dLdI, s));
  return run_adj_g(p, v, nullptr, I, nullptr, 1, p->conv == SRK_ADJ_TRUE, dLdE, s);
}

srk_status op_tangent(const void* f, const void* g, const void* df, const void* dg, const void* gx, const void* gy,
                      int N, int W, int erosion, float dx, srk_stream_t s, void* dh, srk_plan p) {
  const NvtxRange nvtx_range("srk_tangent");
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(dh);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.I = f; a.dI = df; a.out0 = dh;
  return launch_conv_dt<OP_JVP>(p, a, fwd_geom(p, 1), false, s);
}

srk_status op_tangent_adjoint(const void* f, const void* g, const void* df, const void* dg, const void* lam,
                              const void* dlam, const void* gx, const void* gy, int N, int W, int erosion, float dx,
                              srk_stream_t s, void* dLam_f, void* dLam_g, srk_plan p) {
  const NvtxRange nvtx_range("srk_tangent_adjoint");
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(lam);
  SRK_NONNULL(dlam);
  SRK_NONNULL(dLam_f);
  SRK_NONNULL(dLam_g);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  const size_t ww = (size_t)p->W * p->W;
  SRK_TRY(ensure_wbuf(p, 2 * ww * sizeof(float), s));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.v = lam; a.dv = dlam; a.out0 = p->wbuf; a.out1 = p->wbuf + ww;
  SRK_TRY(launch_conv_dt<OP_TANADJ_F>(p, a, fwd_geom(p, 1), false, s));
  SRK_TRY(adj_wrt_f(p, p->wbuf, p->wbuf + ww, nullptr, nullptr, nullptr, 1, dLam_f, s));
  return run_adj_g(p, lam, dlam, f, df, 1, p->conv == SRK_ADJ_TRUE, dLam_g, s);
}

srk_status op_forward(const void* f, const void* g, int B, srk_stream_t s, void* h, srk_plan p) {
  const NvtxRange nvtx_range("srk_forward");
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_TRY(check_batch(p, B));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(h);
  if (!p->have_G) return fail(SRK_ERR_INVALID_ARG, "no kernel set on the plan");
  SRK_TRY(enter(p, s));
  if (p->schedule == SRK_SCHEDULE_DIRECT) return direct_forward(p, g, f, h, B, s);
  OpArgs a = base_args(p);
  a.E = g; a.I = f; a.out0 = h;
  return launch_conv_dt<OP_FWD>(p, a, fwd_geom(p, B), false, s);
}

srk_status op_vjp(const void* v, const void* f, const void* g, int B, srk_stream_t s, void* dLdf, void* dLdg,
                  srk_plan p) {
  const NvtxRange nvtx_range("srk_vjp");
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_TRY(check_batch(p, B));
  SRK_NONNULL(v);
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(dLdf);
  SRK_NONNULL(dLdg);
  if (!p->have_G) return fail(SRK_ERR_INVALID_ARG, "no kernel set on the plan");
  SRK_TRY(enter(p, s));
  const size_t ww = (size_t)p->W * p->W * B;
  SRK_TRY(ensure_wbuf(p, 2 * ww * sizeof(float), s));
  OpArgs a = base_args(p);
  a.E = g; a.v = v; a.out0 = p->wbuf; a.out1 = p->wbuf + ww;
  SRK_TRY(launch_conv_dt<OP_VJP_F>(p, a, fwd_geom(p, B), false, s));
  // per-image wx, wy planes: [B][W][W] each
  SRK_TRY(adj_wrt_f(p, p->wbuf, p->wbuf + ww, nullptr, nullptr, nullptr, B, dLdf, s));
  return run_adj_g(p, v, nullptr, f, nullptr, B, true, dLdg, s);
}

srk_status op_jvp(const void* f, const void* g, const void* df, const void* dg, int B, srk_stream_t s, void* dh,
                  srk_plan p) {
  const NvtxRange nvtx_range("srk_jvp");
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_TRY(check_batch(p, B));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(dh);
  if (!p->have_G) return fail(SRK_ERR_INVALID_ARG, "no kernel set on the plan");
  SRK_TRY(enter(p, s));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.I = f; a.dI = df; a.out0 = dh;
  return launch_conv_dt<OP_JVP>(p, a, fwd_geom(p, B), false, s);
}

// ---- ragged batches -----------------------------------------------------------
// Selects the device tile tables for `key` (the sizes of a ragged batch, or
// a slab's kind, image and columns).  Every key keeps its own tables, built
// on its first call: later calls with any known key upload nothing, so
// calls that alternate keys stay cheap and can be captured in a CUDA graph.
// A key seen for the first time while `s` is being captured is an error
// (building tables copies from host memory, which a graph cannot replay).
// Beyond kMaxTableSets keys the least recently used set is released
// (stream-ordered); a graph captured with it must not be replayed after that.
bool select_tables(srk_plan_s* p, const std::vector<int>& key) {
  auto it = p->tables.find(key);
  if (it == p->tables.end()) return false;
  srk_plan_s::TableSet& t = it->second;
  t.last_use = ++p->table_clock;
  p->rag_tiles = t.tiles;
  p->rag_imgs = t.imgs;
  p->rag_ntiles_fwd = t.ntiles_fwd;
  p->rag_ntiles_adj = t.ntiles_adj;
  p->rag_nblk = t.nblk;
  p->rag_sum_nn = t.sum_nn;
  p->rag_sum_ww = t.sum_ww;
  return true;
}

srk_status missing_tables_in_capture() {
  return fail(SRK_ERR_UNSUPPORTED,
              "ragged/slab tile tables for these sizes are built on their first call, which cannot happen during "
              "stream capture: make one call with the same sizes before capturing");
}

srk_status upload_tables(srk_plan_s* p, std::vector<int> key, std::vector<int4> fwd, const std::vector<int4>& adj,
                         const std::vector<RagImage>& imgs, int nblk, long long sum_nn, long long sum_ww,
                         cudaStream_t s) {
  if (stream_capturing(s)) return missing_tables_in_capture();
  if (p->tables.size() >= srk_plan_s::kMaxTableSets) {
    auto old = p->tables.begin();
    for (auto it = p->tables.begin(); it != p->tables.end(); ++it)
      if (it->second.last_use < old->second.last_use) old = it;
    SRK_CUDA(cudaFreeAsync(old->second.tiles, s));
    SRK_CUDA(cudaFreeAsync(old->second.imgs, s));
    p->tables.erase(old);
  }
  const size_t nt = fwd.size() + adj.size();
  const size_t B = imgs.size();
  srk_plan_s::TableSet t;
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&t.tiles), std::max<size_t>(nt, 1) * sizeof(int4), s));
  const cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&t.imgs), B * sizeof(RagImage), s);
  if (e != cudaSuccess) {
    cudaFreeAsync(t.tiles, s);
    return cuda_status(e, "tile table allocation");
  }
  t.ntiles_fwd = (int)fwd.size();
  t.ntiles_adj = (int)adj.size();
  fwd.insert(fwd.end(), adj.begin(), adj.end());
  // pageable sources: the copies have taken the data when the calls return
  if (nt) SRK_CUDA(cudaMemcpyAsync(t.tiles, fwd.data(), nt * sizeof(int4), cudaMemcpyHostToDevice, s));
  SRK_CUDA(cudaMemcpyAsync(t.imgs, imgs.data(), B * sizeof(RagImage), cudaMemcpyHostToDevice, s));
  t.nblk = nblk;
  t.sum_nn = sum_nn;
  t.sum_ww = sum_ww;
  p->tables[key] = t;
  select_tables(p, key);
  return SRK_OK;
}


// B images of sizes Ns[b] (each 2*erosion+1 <= N_b <= the plan's N; same
// erosion, dx, tile size and spectra), concatenated column-major in every
// buffer: N-sized arrays hold N_b^2 elements per image, W-sized ones W_b^2.
// The tile tables of the forward-type (valid W_b outputs) and adjoint-type
// (N_b outputs) geometries are built together and uploaded once per
// distinct Ns; calls with new sizes re-upload them in stream order.
srk_status ragged_tables(srk_plan_s* p, int B, const int* Ns, cudaStream_t s) {
  if (B < 1) return fail(SRK_ERR_INVALID_ARG, "ragged batch needs B >= 1 (got %d)", B);
  if (!Ns) return fail(SRK_ERR_INVALID_ARG, "Ns is NULL");
  const int e = p->e, S = p->S;
  std::vector<int> key(Ns, Ns + B);
  for (int b = 0; b < B; ++b)
    if (Ns[b] < 2 * e + 1 || Ns[b] > p->N)
      return fail(SRK_ERR_INVALID_ARG, "image %d: N=%d outside [2*erosion+1=%d, plan N=%d]", b, Ns[b], 2 * e + 1, p->N);
  if (select_tables(p, key)) return SRK_OK;
  std::vector<int4> fwd, adj;
  std::vector<RagImage> imgs(B);
  long long on = 0, ow = 0, blk = 0;
  for (int b = 0; b < B; ++b) {
    const int N = Ns[b], W = N - 2 * e;
    imgs[b].on = on;
    imgs[b].ow = ow;
    imgs[b].N = N;
    imgs[b].W = W;
    imgs[b].blk0 = (int)blk;
    imgs[b].cx0 = 0;
    imgs[b].cx1 = N;
    imgs[b].pad = 0;
    on += (long long)N * N;
    ow += (long long)W * W;
    blk += (long long)((N + 31) / 32) * ((N + 8 * kStencilCols - 1) / (8 * kStencilCols));
    const int Tf = (W + S - 1) / S, Ta = (N + S - 1) / S;
    for (int tx = 0; tx < Tf; ++tx)
      for (int ty = 0; ty < Tf; ++ty) fwd.push_back(make_int4(b, tx * S, ty * S, 0));
    for (int tx = 0; tx < Ta; ++tx)
      for (int ty = 0; ty < Ta; ++ty) adj.push_back(make_int4(b, tx * S, ty * S, 0));
  }
  if (blk > (1ll << 30) || fwd.size() + adj.size() > (1u << 30))
    return fail(SRK_ERR_UNSUPPORTED, "ragged batch too large (%lld pixel blocks)", blk);
  return upload_tables(p, std::move(key), std::move(fwd), adj, imgs, (int)blk, on, ow, s);
}

// Column slab [c0, c1) of one N x N image.  Output columns of the
// forward-type geometry (W x W) or, with `adj`, of the adjoint-type one
// (N x N); the tiles start at c0 and step by the tile stride S, so the slab
// spans whole tiles unless it ends at the last output column.  The caller's
// pointers address the slab's first column (column c0 of every array), so
// the image offsets are -c0 columns.
srk_status slab_tables(srk_plan_s* p, int N, int c0, int c1, bool adj, cudaStream_t s) {
  const int e = p->e, S = p->S, W = N - 2 * e;
  if (N < 2 * e + 1 || N > p->N)
    return fail(SRK_ERR_INVALID_ARG, "slab image N=%d outside [2*erosion+1=%d, plan N=%d]", N, 2 * e + 1, p->N);
  const int Wo = adj ? N : W;
  if (c0 < 0 || c1 <= c0 || c1 > Wo)
    return fail(SRK_ERR_INVALID_ARG, "slab columns [%d, %d) outside [0, %d)", c0, c1, Wo);
  if ((c1 - c0) % S != 0 && c1 != Wo)
    return fail(SRK_ERR_INVALID_ARG, "slab [%d, %d) must span whole tiles of %d columns or end at column %d", c0, c1,
                S, Wo);
  std::vector<int> key = {adj ? -2 : -1, N, c0, c1};
  if (select_tables(p, key)) return SRK_OK;
  std::vector<int4> tiles;
  for (int x0 = c0; x0 < c1; x0 += S)
    for (int y0 = 0; y0 < Wo; y0 += S) tiles.push_back(make_int4(0, x0, y0, 0));
  std::vector<RagImage> imgs(1);
  imgs[0].on = -(long long)c0 * N;
  imgs[0].ow = -(long long)c0 * W;
  imgs[0].N = N;
  imgs[0].W = W;
  imgs[0].blk0 = 0;
  imgs[0].cx0 = adj ? c0 : 0;
  imgs[0].cx1 = adj ? c1 : 0;
  imgs[0].pad = 0;
  const int nblk = adj ? ((N + 31) / 32) * ((c1 - c0 + 8 * kStencilCols - 1) / (8 * kStencilCols)) : 0;
  std::vector<int4> none;
  return adj ? upload_tables(p, std::move(key), std::move(none), tiles, imgs, nblk, 0, 0, s)
             : upload_tables(p, std::move(key), std::move(tiles), none, imgs, nblk, 0, 0, s);
}

// The tangent-adjoint on the slab [c0, c1) of the N x N outputs: adjoint-type
// tiles over [c0, c1), and forward-type tiles over the W-columns of its
// intermediate (wx, wy) that the dL/df stencil reads, [c0-e-1, c1-e+1)
// clipped to [0, W): whole tiles from r0 = max(c0-e-1, 0), so the forward-type
// part covers [r0, rE) with rE - r0 a multiple of S (or rE = W).  One image;
// the pointers address column c0 of every array.
srk_status slab_tables_ta(srk_plan_s* p, int N, int c0, int c1, int* r0o, int* rEo, cudaStream_t s) {
  const int e = p->e, S = p->S, W = N - 2 * e;
  if (N < 2 * e + 1 || N > p->N)
    return fail(SRK_ERR_INVALID_ARG, "slab image N=%d outside [2*erosion+1=%d, plan N=%d]", N, 2 * e + 1, p->N);
  if (c0 < 0 || c1 <= c0 || c1 > N) return fail(SRK_ERR_INVALID_ARG, "slab columns [%d, %d) outside [0, %d)", c0, c1, N);
  if ((c1 - c0) % S != 0 && c1 != N)
    return fail(SRK_ERR_INVALID_ARG, "slab [%d, %d) must span whole tiles of %d columns or end at column %d", c0, c1,
                S, N);
  const int r0 = std::max(c0 - e - 1, 0), r1 = std::min(c1 - e + 1, W);
  const int T = r1 > r0 ? (r1 - r0 + S - 1) / S : 0;
  *r0o = r0;
  *rEo = T ? std::min(r0 + T * S, W) : r0;
  std::vector<int> key = {-3, N, c0, c1};
  if (select_tables(p, key)) return SRK_OK;
  std::vector<int4> fwd, adj;
  for (int k = 0; k < T; ++k)
    for (int y0 = 0; y0 < W; y0 += S) fwd.push_back(make_int4(0, r0 + k * S, y0, 0));
  for (int x0 = c0; x0 < c1; x0 += S)
    for (int y0 = 0; y0 < N; y0 += S) adj.push_back(make_int4(0, x0, y0, 0));
  std::vector<RagImage> imgs(1);
  imgs[0].on = -(long long)c0 * N;
  imgs[0].ow = -(long long)c0 * W;
  imgs[0].N = N;
  imgs[0].W = W;
  imgs[0].blk0 = 0;
  imgs[0].cx0 = c0;
  imgs[0].cx1 = c1;
  imgs[0].pad = 0;
  const int nblk = ((N + 31) / 32) * ((c1 - c0 + 8 * kStencilCols - 1) / (8 * kStencilCols));
  return upload_tables(p, std::move(key), std::move(fwd), adj, imgs, nblk, 0, 0, s);
}

Geom ragged_geom(const srk_plan_s* p, bool adj) {
  Geom g = adj ? adj_geom(p, 1) : fwd_geom(p, 1);
  g.U = adj ? p->rag_ntiles_adj : p->rag_ntiles_fwd;
  g.rtile = p->rag_tiles + (adj ? p->rag_ntiles_fwd : 0);
  g.rimg = p->rag_imgs;
  return g;
}

template <typename T>
void adj_wrt_f_rag_t(srk_plan_s* p, const float* wx, const float* wy, const void* v, const void* ux, const void* uy,
                     int B, void* out, cudaStream_t s) {
  const dim3 blk(32, 8);
  if (ux)
    k_adj_wrt_f_rag<T, true><<<p->rag_nblk, blk, 0, s>>>(nullptr, nullptr, static_cast<const T*>(v),
                                                         static_cast<const T*>(ux), static_cast<const T*>(uy),
                                                         p->rag_imgs, B, p->e, static_cast<T*>(out));
  else
    k_adj_wrt_f_rag<T, false><<<p->rag_nblk, blk, 0, s>>>(wx, wy, nullptr, nullptr, nullptr, p->rag_imgs, B, p->e,
                                                          static_cast<T*>(out));
}

srk_status adj_wrt_f_rag(srk_plan_s* p, const float* wx, const float* wy, const void* v, const void* ux,
                         const void* uy, int B, void* out, cudaStream_t s) {
  switch (p->dtype) {
    case SRK_F32: adj_wrt_f_rag_t<float>(p, wx, wy, v, ux, uy, B, out, s); break;
    case SRK_F16: adj_wrt_f_rag_t<__half>(p, wx, wy, v, ux, uy, B, out, s); break;
    case SRK_BF16: adj_wrt_f_rag_t<__nv_bfloat16>(p, wx, wy, v, ux, uy, B, out, s); break;
  }
  return cuda_status(cudaGetLastError(), "ragged adj_wrt_f launch");
}

srk_status check_ragged(const srk_plan_s* p, int erosion, float dx) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  if (erosion != p->e) return fail(SRK_ERR_INVALID_ARG, "erosion=%d differs from the plan's %d", erosion, p->e);
  if (dx != p->dx) return fail(SRK_ERR_INVALID_ARG, "dx=%g differs from the plan's dx=%g", dx, p->dx);
  return SRK_OK;
}

srk_status op_forward_oas_ragged(const void* E, const void* I, const void* gx, const void* gy, int B, const int* Ns,
                                 int erosion, float dx, srk_stream_t s, void* R, srk_plan p) {
  const NvtxRange nvtx_range("srk_forward_oas_ragged");
  SRK_TRY(check_ragged(p, erosion, dx));
  SRK_NONNULL(E);
  SRK_NONNULL(I);
  SRK_NONNULL(R);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(ragged_tables(p, B, Ns, s));
  OpArgs a = base_args(p);
  a.E = E; a.I = I; a.out0 = R;
  return launch_conv_dt<OP_FWD>(p, a, ragged_geom(p, false), false, s);
}

srk_status op_adjoint_ragged(const void* v, const void* ux, const void* uy, const void* I, const void* gx,
                             const void* gy, int B, const int* Ns, int erosion, float dx, srk_stream_t s, void* dLdI,
                             void* dLdE, srk_plan p) {
  const NvtxRange nvtx_range("srk_adjoint_ragged");
  SRK_TRY(check_ragged(p, erosion, dx));
  SRK_NONNULL(v);
  SRK_NONNULL(ux);
  SRK_NONNULL(uy);
  SRK_NONNULL(I);
  SRK_NONNULL(dLdI);
  SRK_NONNULL(dLdE);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(ragged_tables(p, B, Ns, s));
  SRK_TRY(adj_wrt_f_rag(p, nullptr, nullptr, v, ux, uy, B, dLdI, s));
  OpArgs a = base_args(p);
  a.v = v; a.I = I; a.out0 = dLdE;
  return launch_conv_dt<OP_ADJ>(p, a, ragged_geom(p, true), p->conv == SRK_ADJ_TRUE, s);
}

srk_status op_tangent_ragged(const void* f, const void* g, const void* df, const void* dg, const void* gx,
                             const void* gy, int B, const int* Ns, int erosion, float dx, srk_stream_t s, void* dh,
                             srk_plan p) {
  const NvtxRange nvtx_range("srk_tangent_ragged");
  SRK_TRY(check_ragged(p, erosion, dx));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(dh);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(ragged_tables(p, B, Ns, s));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.I = f; a.dI = df; a.out0 = dh;
  return launch_conv_dt<OP_JVP>(p, a, ragged_geom(p, false), false, s);
}

srk_status op_tangent_adjoint_ragged(const void* f, const void* g, const void* df, const void* dg, const void* lam,
                                     const void* dlam, const void* gx, const void* gy, int B, const int* Ns,
                                     int erosion, float dx, srk_stream_t s, void* dLam_f, void* dLam_g, srk_plan p) {
  const NvtxRange nvtx_range("srk_tangent_adjoint_ragged");
  SRK_TRY(check_ragged(p, erosion, dx));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(lam);
  SRK_NONNULL(dlam);
  SRK_NONNULL(dLam_f);
  SRK_NONNULL(dLam_g);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(ragged_tables(p, B, Ns, s));
  const size_t ww = (size_t)p->rag_sum_ww;
  SRK_TRY(ensure_wbuf(p, 2 * ww * sizeof(float), s));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.v = lam; a.dv = dlam; a.out0 = p->wbuf; a.out1 = p->wbuf + ww;
  SRK_TRY(launch_conv_dt<OP_TANADJ_F>(p, a, ragged_geom(p, false), false, s));
  SRK_TRY(adj_wrt_f_rag(p, p->wbuf, p->wbuf + ww, nullptr, nullptr, nullptr, B, dLam_f, s));
  OpArgs b = base_args(p);
  b.v = lam; b.dv = dlam; b.I = f; b.dI = df; b.out0 = dLam_g;
  return launch_conv_dt<OP_ADJ>(p, b, ragged_geom(p, true), p->conv == SRK_ADJ_TRUE, s);
}

// ---- column slabs of one image ------------------------------------------------
srk_status op_forward_oas_slab(const void* E, const void* I, const void* gx, const void* gy, int N, int erosion,
                               float dx, int c0, int c1, srk_stream_t s, void* R, srk_plan p) {
  const NvtxRange nvtx_range("srk_forward_oas_slab");
  SRK_TRY(check_ragged(p, erosion, dx));
  SRK_NONNULL(E);
  SRK_NONNULL(I);
  SRK_NONNULL(R);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(slab_tables(p, N, c0, c1, false, s));
  OpArgs a = base_args(p);
  a.E = E; a.I = I; a.out0 = R;
  return launch_conv_dt<OP_FWD>(p, a, ragged_geom(p, false), false, s);
}

srk_status op_tangent_slab(const void* f, const void* g, const void* df, const void* dg, const void* gx,
                           const void* gy, int N, int erosion, float dx, int c0, int c1, srk_stream_t s, void* dh,
                           srk_plan p) {
  const NvtxRange nvtx_range("srk_tangent_slab");
  SRK_TRY(check_ragged(p, erosion, dx));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(dh);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(slab_tables(p, N, c0, c1, false, s));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.I = f; a.dI = df; a.out0 = dh;
  return launch_conv_dt<OP_JVP>(p, a, ragged_geom(p, false), false, s);
}

srk_status op_adjoint_slab(const void* v, const void* ux, const void* uy, const void* I, const void* gx,
                           const void* gy, int N, int erosion, float dx, int c0, int c1, srk_stream_t s, void* dLdI,
                           void* dLdE, srk_plan p) {
  const NvtxRange nvtx_range("srk_adjoint_slab");
  SRK_TRY(check_ragged(p, erosion, dx));
  SRK_NONNULL(v);
  SRK_NONNULL(ux);
  SRK_NONNULL(uy);
  SRK_NONNULL(I);
  SRK_NONNULL(dLdI);
  SRK_NONNULL(dLdE);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(slab_tables(p, N, c0, c1, true, s));
  SRK_TRY(adj_wrt_f_rag(p, nullptr, nullptr, v, ux, uy, 1, dLdI, s));
  OpArgs a = base_args(p);
  a.v = v; a.I = I; a.out0 = dLdE;
  return launch_conv_dt<OP_ADJ>(p, a, ragged_geom(p, true), p->conv == SRK_ADJ_TRUE, s);
}

srk_status op_tangent_adjoint_slab(const void* f, const void* g, const void* df, const void* dg, const void* lam,
                                   const void* dlam, const void* gx, const void* gy, int N, int erosion, float dx,
                                   int c0, int c1, srk_stream_t s, void* dLam_f, void* dLam_g, srk_plan p) {
  const NvtxRange nvtx_range("srk_tangent_adjoint_slab");
  SRK_TRY(check_ragged(p, erosion, dx));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(lam);
  SRK_NONNULL(dlam);
  SRK_NONNULL(dLam_f);
  SRK_NONNULL(dLam_g);
  SRK_TRY(enter(p, s));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  int r0 = 0, rE = 0;
  SRK_TRY(slab_tables_ta(p, N, c0, c1, &r0, &rE, s));
  const int W = N - 2 * p->e;
  const size_t ww = (size_t)(rE - r0) * W;
  SRK_TRY(ensure_wbuf(p, std::max<size_t>(2 * ww, 1) * sizeof(float), s));
  // wx, wy hold the W-columns [r0, rE); their pointers address column c0
  float* wx = p->wbuf + (ptrdiff_t)(c0 - r0) * W;
  float* wy = wx + ww;
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.v = lam; a.dv = dlam; a.out0 = wx; a.out1 = wy;
  SRK_TRY(launch_conv_dt<OP_TANADJ_F>(p, a, ragged_geom(p, false), false, s));
  SRK_TRY(adj_wrt_f_rag(p, wx, wy, nullptr, nullptr, nullptr, 1, dLam_f, s));
  OpArgs b = base_args(p);
  b.v = lam; b.dv = dlam; b.I = f; b.dI = df; b.out0 = dLam_g;
  return launch_conv_dt<OP_ADJ>(p, b, ragged_geom(p, true), p->conv == SRK_ADJ_TRUE, s);
}

// The float* entry points are the reference drop-ins: fp32 plans only.
srk_status need_f32(srk_plan p) {
  if (p && p->dtype != SRK_F32)
    return fail(SRK_ERR_INVALID_ARG, "this entry point takes float buffers; the plan stores dtype %d (use the _t form)",
                (int)p->dtype);
  return SRK_OK;
}

}  // namespace
extern "C" {

srk_status srk_training_forward(const float* E, const float* I, const void* gx, const void* gy, int N, int W,
                                int erosion, float dx, int B, srk_stream_t s, float* R, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_training_forward(E, I, gx, gy, N, W, erosion, dx, B, s, R, p);
}

srk_status srk_training_forward_sync(const float* E, const float* I, const void* gx, const void* gy, int N, int W,
                                     int erosion, float dx, int B, srk_stream_t s, float* R, srk_plan p) {
  SRK_TRY(srk_training_forward(E, I, gx, gy, N, W, erosion, dx, B, s, R, p));
  return srk_plan_sync(p, s);
}

srk_status srk_forward_oas(const float* E, const float* I, const void* gx, const void* gy, int N, int W,
                           int erosion, float dx, srk_stream_t s, float* R, srk_plan p, float* ux, float* uy) {
  SRK_TRY(need_f32(p));
  return op_forward_oas(E, I, gx, gy, N, W, erosion, dx, s, R, p, ux, uy);
}

srk_status srk_adjoint(const float* v, const float* ux, const float* uy, const float* I, const void* gx,
                       const void* gy, int N, int W, int erosion, float dx, srk_stream_t s, float* dLdI, float* dLdE,
                       srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_adjoint(v, ux, uy, I, gx, gy, N, W, erosion, dx, s, dLdI, dLdE, p);
}

srk_status srk_tangent(const float* f, const float* g, const float* df, const float* dg, const void* gx,
                       const void* gy, int N, int W, int erosion, float dx, srk_stream_t s, float* dh, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_tangent(f, g, df, dg, gx, gy, N, W, erosion, dx, s, dh, p);
}

srk_status srk_tangent_adjoint(const float* f, const float* g, const float* df, const float* dg, const float* lam,
                               const float* dlam, const void* gx, const void* gy, int N, int W, int erosion, float dx,
                               srk_stream_t s, float* dLam_f, float* dLam_g, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_tangent_adjoint(f, g, df, dg, lam, dlam, gx, gy, N, W, erosion, dx, s, dLam_f, dLam_g, p);
}

srk_status srk_forward(const float* f, const float* g, int B, srk_stream_t s, float* h, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_forward(f, g, B, s, h, p);
}

srk_status srk_vjp(const float* v, const float* f, const float* g, int B, srk_stream_t s, float* dLdf, float* dLdg,
                   srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_vjp(v, f, g, B, s, dLdf, dLdg, p);
}

srk_status srk_jvp(const float* f, const float* g, const float* df, const float* dg, int B, srk_stream_t s,
                   float* dh, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_jvp(f, g, df, dg, B, s, dh, p);
}

srk_status srk_forward_oas_slab(const float* E, const float* I, const void* gx, const void* gy, int N, int erosion,
                                float dx, int c0, int c1, srk_stream_t s, float* R, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_forward_oas_slab(E, I, gx, gy, N, erosion, dx, c0, c1, s, R, p);
}

srk_status srk_tangent_slab(const float* f, const float* g, const float* df, const float* dg, const void* gx,
                            const void* gy, int N, int erosion, float dx, int c0, int c1, srk_stream_t s, float* dh,
                            srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_tangent_slab(f, g, df, dg, gx, gy, N, erosion, dx, c0, c1, s, dh, p);
}

srk_status srk_adjoint_slab(const float* v, const float* ux, const float* uy, const float* I, const void* gx,
                            const void* gy, int N, int erosion, float dx, int c0, int c1, srk_stream_t s,
                            float* dLdI, float* dLdE, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_adjoint_slab(v, ux, uy, I, gx, gy, N, erosion, dx, c0, c1, s, dLdI, dLdE, p);
}

srk_status srk_tangent_adjoint_slab(const float* f, const float* g, const float* df, const float* dg,
                                    const float* lam, const float* dlam, const void* gx, const void* gy, int N,
                                    int erosion, float dx, int c0, int c1, srk_stream_t s, float* dLam_f,
                                    float* dLam_g, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_tangent_adjoint_slab(f, g, df, dg, lam, dlam, gx, gy, N, erosion, dx, c0, c1, s, dLam_f, dLam_g, p);
}

srk_status srk_forward_oas_ragged(const float* E, const float* I, const void* gx, const void* gy, int B,
                                  const int* Ns, int erosion, float dx, srk_stream_t s, float* R, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_forward_oas_ragged(E, I, gx, gy, B, Ns, erosion, dx, s, R, p);
}

srk_status srk_adjoint_ragged(const float* v, const float* ux, const float* uy, const float* I, const void* gx,
                              const void* gy, int B, const int* Ns, int erosion, float dx, srk_stream_t s,
                              float* dLdI, float* dLdE, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_adjoint_ragged(v, ux, uy, I, gx, gy, B, Ns, erosion, dx, s, dLdI, dLdE, p);
}

srk_status srk_tangent_ragged(const float* f, const float* g, const float* df, const float* dg, const void* gx,
                              const void* gy, int B, const int* Ns, int erosion, float dx, srk_stream_t s, float* dh,
                              srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_tangent_ragged(f, g, df, dg, gx, gy, B, Ns, erosion, dx, s, dh, p);
}

srk_status srk_tangent_adjoint_ragged(const float* f, const float* g, const float* df, const float* dg,
                                      const float* lam, const float* dlam, const void* gx, const void* gy, int B,
                                      const int* Ns, int erosion, float dx, srk_stream_t s, float* dLam_f,
                                      float* dLam_g, srk_plan p) {
  SRK_TRY(need_f32(p));
  return op_tangent_adjoint_ragged(f, g, df, dg, lam, dlam, gx, gy, B, Ns, erosion, dx, s, dLam_f, dLam_g, p);
}

// ---- storage-typed forms: element type of every image buffer = plan dtype ------
srk_status srk_training_forward_t(const void* E, const void* I, const void* gx, const void* gy, int N, int W,
                                  int erosion, float dx, int B, srk_stream_t s, void* R, srk_plan p) {
  return op_training_forward(E, I, gx, gy, N, W, erosion, dx, B, s, R, p);
}
srk_status srk_forward_oas_t(const void* E, const void* I, const void* gx, const void* gy, int N, int W, int erosion,
                             float dx, srk_stream_t s, void* R, srk_plan p, void* ux, void* uy) {
  return op_forward_oas(E, I, gx, gy, N, W, erosion, dx, s, R, p, ux, uy);
}
srk_status srk_adjoint_t(const void* v, const void* ux, const void* uy, const void* I, const void* gx, const void* gy,
                         int N, int W, int erosion, float dx, srk_stream_t s, void* dLdI, void* dLdE, srk_plan p) {
  return op_adjoint(v, ux, uy, I, gx, gy, N, W, erosion, dx, s, dLdI, dLdE, p);
}
srk_status srk_tangent_t(const void* f, const void* g, const void* df, const void* dg, const void* gx, const void* gy,
                         int N, int W, int erosion, float dx, srk_stream_t s, void* dh, srk_plan p) {
  return op_tangent(f, g, df, dg, gx, gy, N, W, erosion, dx, s, dh, p);
}
srk_status srk_tangent_adjoint_t(const void* f, const void* g, const void* df, const void* dg, const void* lam,
                                 const void* dlam, const void* gx, const void* gy, int N, int W, int erosion,
                                 float dx, srk_stream_t s, void* dLam_f, void* dLam_g, srk_plan p) {
  return op_tangent_adjoint(f, g, df, dg, lam, dlam, gx, gy, N, W, erosion, dx, s, dLam_f, dLam_g, p);
}
srk_status srk_forward_t(const void* f, const void* g, int B, srk_stream_t s, void* h, srk_plan p) {
  return op_forward(f, g, B, s, h, p);
}
srk_status srk_vjp_t(const void* v, const void* f, const void* g, int B, srk_stream_t s, void* dLdf, void* dLdg,
                     srk_plan p) {
  return op_vjp(v, f, g, B, s, dLdf, dLdg, p);
}
srk_status srk_jvp_t(const void* f, const void* g, const void* df, const void* dg, int B, srk_stream_t s, void* dh,
                     srk_plan p) {
  return op_jvp(f, g, df, dg, B, s, dh, p);
}

srk_status srk_autotune(int N, int W, int erosion, float dx, int B, srk_dtype dtype, int* tile_M, int* schedule) {
  if (!tile_M || !schedule) return fail(SRK_ERR_INVALID_ARG, "NULL output pointer");
  if (N < 3 || erosion < 0 || W != N - 2 * erosion || W < 1 || B < 1)
    return fail(SRK_ERR_INVALID_ARG, "bad sizes for autotune (N=%d W=%d erosion=%d B=%d)", N, W, erosion, B);
  const std::string key = tune_key(N, W, erosion, B, dtype);
  if (tune_lookup(key, tile_M, schedule)) return SRK_OK;
  // synthetic workload: a smooth Green's tensor and uniform images
  const int KW = 2 * erosion + 1;
  const int Bt = B < 512 ? B : 512;
  const size_t esz = dtype == SRK_F32 ? 4 : 2;
  cudaStream_t s = nullptr;
  SRK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  float *Kx = nullptr, *Ky = nullptr;
  void *E = nullptr, *R = nullptr;
  srk_status st = SRK_OK;
  float best = 0.f;
  int bestM = 0, bestS = SRK_SCHEDULE_THREE_PASS;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto done = [&](srk_status r) {
    if (Kx) cudaFree(Kx);
    if (Ky) cudaFree(Ky);
    if (E) cudaFree(E);
    if (R) cudaFree(R);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    return r;
  };
  if (cudaMalloc(&Kx, sizeof(float) * KW * KW) != cudaSuccess || cudaMalloc(&Ky, sizeof(float) * KW * KW) != cudaSuccess ||
      cudaMalloc(&E, esz * (size_t)Bt * N * N) != cudaSuccess || cudaMalloc(&R, esz * (size_t)Bt * W * W) != cudaSuccess)
    return done(fail(SRK_ERR_ALLOC, "autotune buffers"));
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  if ((st = srk_green_tensor(Kx, Ky, KW, 1.0 / (erosion / 3.0 + 1.0), (double)erosion + 0.5, 1.0, s)) != SRK_OK)
    return done(st);
  // any bit pattern is a valid half input too; the values only need to be finite
  k_fill_pattern<<<256, 256, 0, s>>>(static_cast<float*>(E), esz * (size_t)Bt * N * N / 4, 1234u);
  if (dtype != SRK_F32) SRK_CUDA(cudaMemsetAsync(E, 0, esz * (size_t)Bt * N * N, s));
  const int cand[3] = {128, 256, 512};
  for (int M : cand) {
    if (M - 2 * erosion < 16) continue;
    for (int sch = 0; sch < 2; ++sch) {
      srk_plan p = nullptr;
      if (srk_plan_create(&p, N, W, erosion, dx, Bt, N + (N & 1), dtype, M, 0) != SRK_OK) continue;
      p->schedule = sch;
      p->persist_prefetch = 0;
      if ((st = srk_plan_set_kernel(p, Kx, Ky, KW, s)) != SRK_OK) { srk_plan_destroy(p); return done(st); }
      for (int it = 0; it < 2; ++it) op_forward(E, E, Bt, s, R, p);
      cudaEventRecord(e0, s);
      for (int it = 0; it < 3; ++it) op_forward(E, E, Bt, s, R, p);
      cudaEventRecord(e1, s);
      st = srk_plan_sync(p, s);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      srk_plan_destroy(p);
      if (st != SRK_OK) return done(st);
      if (bestM == 0 || ms < best) { best = ms; bestM = M; bestS = sch; }
    }
  }
  if (bestM == 0) return done(fail(SRK_ERR_UNSUPPORTED, "no tile size fits erosion=%d", erosion));
  {
    // the tensor-core direct schedule of the forward, where it applies
    srk_plan p = nullptr;
    if (srk_plan_create(&p, N, W, erosion, dx, Bt, N + (N & 1), dtype, bestM, 0) == SRK_OK) {
      std::string why;
      if (direct_supported(p, N, &why) && srk_plan_set_schedule(p, SRK_SCHEDULE_DIRECT) == SRK_OK &&
          (st = srk_plan_set_kernel(p, Kx, Ky, KW, s)) == SRK_OK) {
        for (int it = 0; it < 2; ++it) op_forward(E, E, Bt, s, R, p);
        cudaEventRecord(e0, s);
        for (int it = 0; it < 3; ++it) op_forward(E, E, Bt, s, R, p);
        cudaEventRecord(e1, s);
        st = srk_plan_sync(p, s);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (st == SRK_OK && ms < best) {
          best = ms;
          bestS = SRK_SCHEDULE_DIRECT;
        }
      }
      srk_plan_destroy(p);
      if (st != SRK_OK) return done(st);
    }
  }
  if (dtype != SRK_F32 && 512 - 2 * erosion >= 16) {
    // the tensor-core row pass (tile 512), where it applies
    srk_plan p = nullptr;
    if (srk_plan_create(&p, N, W, erosion, dx, Bt, N + (N & 1), dtype, 512, 0) == SRK_OK) {
      std::string why;
      if (tensor_rows_supported(p, &why) && srk_plan_set_schedule(p, SRK_SCHEDULE_TENSOR_ROWS) == SRK_OK &&
          (st = srk_plan_set_kernel(p, Kx, Ky, KW, s)) == SRK_OK) {
        for (int it = 0; it < 2; ++it) op_forward(E, E, Bt, s, R, p);
        cudaEventRecord(e0, s);
        for (int it = 0; it < 3; ++it) op_forward(E, E, Bt, s, R, p);
        cudaEventRecord(e1, s);
        st = srk_plan_sync(p, s);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (st == SRK_OK && ms < best) {
          best = ms;
          bestM = 512;
          bestS = SRK_SCHEDULE_TENSOR_ROWS;
        }
      }
      srk_plan_destroy(p);
      if (st != SRK_OK) return done(st);
    }
  }
  *tile_M = bestM;
  *schedule = bestS;
  tune_store(key, bestM, bestS);
  return done(SRK_OK);
}

}  // extern "C"
