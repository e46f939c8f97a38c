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
#include <string>
#include <vector>

#include "../../include/srk_b200.h"
#include "engine.cuh"
#include "spectra.cuh"

using namespace srk;

namespace {

thread_local std::string g_last_error;

srk_status fail(srk_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

srk_status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SRK_OK;
  return fail(e == cudaErrorMemoryAllocation ? SRK_ERR_ALLOC : SRK_ERR_CUDA, "%s: %s", what,
              cudaGetErrorString(e));
}

#define SRK_TRY(expr)                        \
  do {                                       \
    const srk_status _s = (expr);            \
    if (_s != SRK_OK) return _s;             \
  } while (0)
#define SRK_CUDA(expr) SRK_TRY(cuda_status((expr), #expr))


// Host double-precision twiddle table (cos, sin)(2 pi m / M).
std::vector<double2> twiddles64(int M) {
  std::vector<double2> t(M);
  for (int m = 0; m < M; ++m) {
    const double a = 2.0 * 3.14159265358979323846 * (double)m / (double)M;
    t[m] = make_double2(std::cos(a), std::sin(a));
  }
  return t;
}

}  // namespace

struct srk_plan_s {
  int device = 0;
  int N = 0, W = 0, e = 0, B_max = 0, spectra_M = 0;
  float dx = 1.f;
  srk_dtype dtype = SRK_F32;
  srk_adj_convention conv = SRK_ADJ_REFERENCE;
  int M = 0, S = 0, T = 0, Ta = 0;
  int chunk = 0;
  float2* G[2] = {nullptr, nullptr};   // engine-layout spectra, scaled by 1/M^2
  bool have_G = false;
  const void* src[2] = {nullptr, nullptr};
  float2* tw = nullptr;                // W_M^m, float
  float2* scratch = nullptr;
  size_t scratch_bytes = 0;
  float* wbuf = nullptr;               // wx, wy for dL/df
  size_t wbuf_bytes = 0;
  int schedule = SRK_SCHEDULE_PERSISTENT;
  Ctl* ctl = nullptr;                  // persistent-kernel control block
  unsigned int* mailbox = nullptr;     // pinned host copy of (abort, where)
  cudaEvent_t mailbox_ev = nullptr;
  bool mailbox_pending = false;
  unsigned long long spin_limit = 1ull << 25;
  unsigned long long* mailbox_spins = nullptr;  // pinned: spin polls of the last launch
  int persist_lag = 0, persist_grid = 0, persist_prefetch = 1;
  int last_grid = 0, last_launches = 0, last_lag = 0, last_nslot = 0;
};

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
  g.M = p->M; g.e = p->e; g.S = p->S; g.T = p->T;
  g.Nin = p->N; g.Wout = p->W; g.TT = p->T * p->T; g.U = B * g.TT;
  return g;
}
Geom adj_geom(const srk_plan_s* p, int B) {
  Geom g;
  g.M = p->M; g.e = p->e; g.S = p->S; g.T = p->Ta;
  g.Nin = p->N + 2 * p->e; g.Wout = p->N; g.TT = p->Ta * p->Ta; g.U = B * g.TT;
  return g;
}

size_t wt_bytes(int M, int S) {
  const size_t P = (size_t)s2_pitch(S);
  const size_t fwd = (size_t)M * M + 2 * P * M;
  const size_t adj = 2 * (size_t)M * M + P * M;
  return sizeof(float2) * (fwd > adj ? fwd : adj);
}

// ---- launch helpers -------------------------------------------------------------
template <typename K>
srk_status set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024)
    SRK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return SRK_OK;
}

template <int M, int OP, typename T>
srk_status launch_conv_m(srk_plan_s* p, const OpArgs& a, const Geom& g, int nwt, bool conjG, cudaStream_t s) {
  constexpr int K = OpTraits<OP>::K;
  constexpr int L = OpTraits<OP>::L;
  const size_t sm1 = phase_smem_bytes<M>();
  const size_t sm2 = sm1;
  const size_t sm3 = sm1;
  const size_t per = wt_elems<M, OP>(g.S);
  const size_t cap = p->scratch_bytes / sizeof(float2) / per;  // WTs that fit the scratch
  if (p->schedule == SRK_SCHEDULE_PERSISTENT && cap >= 3) {
    SRK_TRY(set_smem(k_persist<M, OP, T>, sm2));
    int dev = 0, nsm = 0, per_sm = 0;
    SRK_CUDA(cudaGetDevice(&dev));
    SRK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    SRK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist<M, OP, T>, kThreads, sm2));
    if (per_sm < 1) return fail(SRK_ERR_UNSUPPORTED, "persistent kernel does not fit an SM (smem %zu)", sm2);
    const int round = M / kWarps * 2 + (g.S + kWarps - 1) / kWarps;
    int grid = nsm * per_sm;
    if (p->persist_grid > 0) grid = std::min(grid, p->persist_grid);
    // Tickets in flight ~ grid (x2 with prefetch): the lag between the phases
    // of a WT must exceed that window so a unit rarely finds its
    // dependency unmet; the ring must hold 2*lag+2 WTs for the same reason.
    const int window = grid * (p->persist_prefetch ? 2 : 1);
    PersistParams pp;
    pp.lag = p->persist_lag > 0 ? p->persist_lag : (window + round - 1) / round + 1;
    pp.nslot = 2 * pp.lag + 2;
    pp.prefetch = p->persist_prefetch;
    pp.pad = 0;
    pp.spin_limit = p->spin_limit;
    if (pp.nslot > (int)std::min<size_t>(cap, kMaxSlots)) {
      pp.nslot = (int)std::min<size_t>(cap, kMaxSlots);
      pp.lag = std::min(pp.lag, pp.nslot - 1);
    }
    const long long tickets = (long long)(nwt + 2 * pp.lag) * round;
    grid = (int)std::min<long long>(grid, tickets);
    SRK_CUDA(cudaMemsetAsync(p->ctl, 0, sizeof(Ctl), s));
    k_persist<M, OP, T><<<grid, kThreads, sm2, s>>>(a, g, p->G[0], p->G[1], conjG ? 1 : 0, p->tw, p->scratch, nwt,
                                                   p->ctl, pp);
    SRK_CUDA(cudaGetLastError());
    SRK_CUDA(cudaMemcpyAsync(p->mailbox, &p->ctl->abort, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    SRK_CUDA(cudaMemcpyAsync(p->mailbox_spins, &p->ctl->spins, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             s));
    SRK_CUDA(cudaEventRecord(p->mailbox_ev, s));
    p->mailbox_pending = true;
    p->last_grid = grid;
    p->last_launches = 1;
    p->last_lag = pp.lag;
    p->last_nslot = pp.nslot;
    return SRK_OK;
  }
  SRK_TRY(set_smem(k_p1<M, OP, T>, sm1));
  SRK_TRY(set_smem(k_p2<M, OP>, sm2));
  SRK_TRY(set_smem(k_p3<M, OP, T>, sm3));
  const int chunk = (int)std::min<size_t>(std::max<size_t>(cap, 1), 65535);
  int launches = 0;
  for (int w0 = 0; w0 < nwt; w0 += chunk) {
    const int c = (nwt - w0 < chunk) ? (nwt - w0) : chunk;
    k_p1<M, OP, T><<<dim3(M / kWarps, c), kThreads, sm1, s>>>(a, g, p->tw, w0, p->scratch, g.S);
    k_p2<M, OP><<<dim3(M / kWarps, c), kThreads, sm2, s>>>(p->scratch, p->G[0], p->G[1], conjG ? 1 : 0, g, p->tw);
    k_p3<M, OP, T><<<dim3((g.S + kWarps - 1) / kWarps, c), kThreads, sm3, s>>>(p->scratch, a, g, p->tw, w0);
    launches += 3;
  }
  p->last_launches = launches;
  return cuda_status(cudaGetLastError(), "conv launch");
}

template <int OP, typename T>
srk_status launch_conv(srk_plan_s* p, const OpArgs& a, const Geom& g, bool conjG, cudaStream_t s) {
  const int nwt = OpTraits<OP>::PAIRS ? (g.U + 1) / 2 : g.U;
  if (nwt <= 0) return SRK_OK;
  switch (p->M) {
    case 128: return launch_conv_m<128, OP, T>(p, a, g, nwt, conjG, s);
    case 256: return launch_conv_m<256, OP, T>(p, a, g, nwt, conjG, s);
    case 512: return launch_conv_m<512, OP, T>(p, a, g, nwt, conjG, s);
    default: return fail(SRK_ERR_UNSUPPORTED, "tile size %d not built", p->M);
  }
}

srk_status ensure_wbuf(srk_plan_s* p, size_t bytes, cudaStream_t s) {
  if (p->wbuf_bytes >= bytes) return SRK_OK;
  if (p->wbuf) SRK_CUDA(cudaFreeAsync(p->wbuf, s));
  p->wbuf = nullptr;
  p->wbuf_bytes = 0;
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p->wbuf), bytes, s));
  p->wbuf_bytes = bytes;
  return SRK_OK;
}

srk_status adj_wrt_f(srk_plan_s* p, const float* wx, const float* wy, const float* v, const float* ux,
                     const float* uy, int B, float* out, cudaStream_t s) {
  const dim3 blk(32, 8);
  const dim3 grd((p->N + 31) / 32, (p->N + 7) / 8, B);
  if (ux)
    k_adj_wrt_f<float, true><<<grd, blk, 0, s>>>(nullptr, nullptr, v, ux, uy, p->N, p->W, p->e, B, out);
  else
    k_adj_wrt_f<float, false><<<grd, blk, 0, s>>>(wx, wy, nullptr, nullptr, nullptr, p->N, p->W, p->e, B, out);
  return cuda_status(cudaGetLastError(), "adj_wrt_f launch");
}

// ---- spectra -----------------------------------------------------------------------
srk_status upload_table(const std::vector<double2>& t, double2** d, cudaStream_t s) {
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(d), t.size() * sizeof(double2), s));
  SRK_CUDA(cudaMemcpyAsync(*d, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
  // the host vector dies with this call: make the copy complete first
  SRK_CUDA(cudaStreamSynchronize(s));
  return SRK_OK;
}

// Spatial kernel (double, column-major KW x KW) -> engine spectrum at size M.
srk_status spectrum_from_spatial(const double* Kd, int KW, int M, double scale, float2* full, float2* ref,
                                 cudaStream_t s) {
  double2* tab = nullptr;
  double2* P = nullptr;
  SRK_TRY(upload_table(twiddles64(M), &tab, s));
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&P), sizeof(double2) * (size_t)KW * M, s));
  k_dft_cols<<<dim3((M + 127) / 128, KW), 128, 0, s>>>(Kd, KW, M, tab, P);
  k_dft_rows<<<dim3((M + 127) / 128, M), 128, 0, s>>>(P, KW, M, tab, scale, full, ref);
  SRK_CUDA(cudaGetLastError());
  SRK_CUDA(cudaFreeAsync(P, s));
  SRK_CUDA(cudaFreeAsync(tab, s));
  return SRK_OK;
}

srk_status import_one(srk_plan_s* p, const float2* ref, float2* full, cudaStream_t s) {
  const int Mr = p->spectra_M;
  // dx^2 / M^2 folded into the spectrum (srkConvOaS applies dx*dx/(M*M), srk_forward.cuh:380)
  const float scale = (p->dx * p->dx) / ((float)p->M * (float)p->M);
  if (Mr == p->M) {
    k_relayout<<<dim3((Mr + 127) / 128, Mr), 128, 0, s>>>(ref, Mr, scale, full);
    return cuda_status(cudaGetLastError(), "relayout");
  }
  // Different FFT size: recover the spatial kernel on its (2e+1)^2 support in
  // FP64, then take its spectrum at the tile size.
  const int c = p->e;
  const int KW = 2 * c + 1;
  double2* tab = nullptr;
  double2* Tm = nullptr;
  double* Kd = nullptr;
  SRK_TRY(upload_table(twiddles64(Mr), &tab, s));
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&Tm), sizeof(double2) * (size_t)(Mr / 2 + 1) * KW, s));
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&Kd), sizeof(double) * (size_t)KW * KW, s));
  k_recover_a<<<dim3((KW + 127) / 128, Mr / 2 + 1), 128, 0, s>>>(ref, Mr, c, tab, Tm);
  k_recover_b<<<(KW * KW + 127) / 128, 128, 0, s>>>(Tm, Mr, c, tab, Kd);
  SRK_CUDA(cudaGetLastError());
  SRK_TRY(spectrum_from_spatial(Kd, KW, p->M, (double)scale, full, nullptr, s));
  SRK_CUDA(cudaFreeAsync(Tm, s));
  SRK_CUDA(cudaFreeAsync(Kd, s));
  SRK_CUDA(cudaFreeAsync(tab, s));
  return SRK_OK;
}

srk_status import_spectra(srk_plan_s* p, const void* gx, const void* gy, cudaStream_t s) {
  if (!gx || !gy) return fail(SRK_ERR_INVALID_ARG, "kernel spectra are NULL");
  SRK_TRY(import_one(p, static_cast<const float2*>(gx), p->G[0], s));
  SRK_TRY(import_one(p, static_cast<const float2*>(gy), p->G[1], s));
  p->src[0] = gx;
  p->src[1] = gy;
  p->have_G = true;
  return SRK_OK;
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

srk_status enter(srk_plan_s* p) {
  SRK_TRY(set_device(p));
  return check_mailbox(p);
}

// dL/dg through the adjoint engine: h = v*df (+ dv*f' for the tangent-adjoint)
srk_status run_adj_g(srk_plan_s* p, const float* v, const float* dv, const float* f, const float* df, int B,
                     bool conj, float* out, cudaStream_t s) {
  OpArgs a = base_args(p);
  a.v = v; a.dv = dv; a.I = f; a.dI = df; a.out0 = out;
  return launch_conv<OP_ADJ, float>(p, a, adj_geom(p, B), conj, s);
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
  if (dtype != SRK_F32) return fail(SRK_ERR_UNSUPPORTED, "dtype %d: only SRK_F32 plans in this build", (int)dtype);
  if (!(dx > 0.f) || !std::isfinite(dx)) return fail(SRK_ERR_INVALID_ARG, "dx=%g must be positive", dx);
  int M = tile_M;
  if (M == 0) M = choose_tile(N, W, erosion);
  if (M == 0)
    return fail(SRK_ERR_UNSUPPORTED, "erosion=%d too large for the 512 tile (needs stride >= 16)", erosion);
  if (!(M == 128 || M == 256 || M == 512)) return fail(SRK_ERR_INVALID_ARG, "tile_M=%d not in {128,256,512}", M);
  if (M - 2 * erosion < 8) return fail(SRK_ERR_UNSUPPORTED, "tile_M=%d leaves no valid stride for erosion=%d", M, erosion);

  srk_plan_s* p = new srk_plan_s();
  cudaGetDevice(&p->device);
  p->N = N; p->W = W; p->e = erosion; p->dx = dx; p->B_max = B_max; p->spectra_M = spectra_M; p->dtype = dtype;
  p->M = M; p->S = M - 2 * erosion;
  p->T = (W + p->S - 1) / p->S;
  p->Ta = (N + p->S - 1) / p->S;
  const size_t nwt_max = std::max<size_t>({(size_t)(B_max * (size_t)p->T * p->T + 1) / 2,
                                           (size_t)B_max * p->T * p->T,
                                           (size_t)(B_max * (size_t)p->Ta * p->Ta + 1) / 2});
  const size_t per = wt_bytes(M, p->S);
  const size_t cap = budget ? budget : ((size_t)1 << 30);
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
  std::vector<float2> tw(M);
  const std::vector<double2> t64 = twiddles64(M);
  for (int m = 0; m < M; ++m) tw[m] = make_float2((float)t64[m].x, (float)-t64[m].y);  // exp(-2 pi i m/M)
  if ((err = cudaMemcpy(p->tw, tw.data(), sizeof(float2) * M, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cleanup(cuda_status(err, "twiddle upload"));
  *out = p;
  return SRK_OK;
}

srk_status srk_plan_destroy(srk_plan p) {
  if (!p) return SRK_OK;
  cudaSetDevice(p->device);
  cudaDeviceSynchronize();
  if (p->scratch) cudaFree(p->scratch);
  if (p->G[0]) cudaFree(p->G[0]);
  if (p->G[1]) cudaFree(p->G[1]);
  if (p->tw) cudaFree(p->tw);
  if (p->wbuf) cudaFree(p->wbuf);
  if (p->ctl) cudaFree(p->ctl);
  if (p->mailbox) cudaFreeHost(p->mailbox);
  if (p->mailbox_spins) cudaFreeHost(p->mailbox_spins);
  if (p->mailbox_ev) cudaEventDestroy(p->mailbox_ev);
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
  if (sch != SRK_SCHEDULE_PERSISTENT && sch != SRK_SCHEDULE_THREE_PASS)
    return fail(SRK_ERR_INVALID_ARG, "bad schedule %d", (int)sch);
  p->schedule = sch;
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
  return check_mailbox(p);
}

srk_status srk_debug_wait_selftest(srk_plan p, unsigned long long spin_limit, srk_stream_t s) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  if (spin_limit == 0 || spin_limit > (1ull << 26)) return fail(SRK_ERR_INVALID_ARG, "spin_limit out of range");
  SRK_TRY(enter(p));
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
  double* Kd = nullptr;
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&Kd), sizeof(double) * KW * KW, s));
  const double scale = (double)p->dx * (double)p->dx / ((double)p->M * (double)p->M);
  const float* K[2] = {Kx, Ky};
  for (int i = 0; i < 2; ++i) {
    k_float_to_double<<<(KW * KW + 255) / 256, 256, 0, s>>>(K[i], Kd, KW * KW);
    SRK_TRY(spectrum_from_spatial(Kd, KW, p->M, scale, p->G[i], nullptr, s));
  }
  SRK_CUDA(cudaFreeAsync(Kd, s));
  p->src[0] = p->src[1] = nullptr;
  p->have_G = true;
  return SRK_OK;
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
  double* Kd = nullptr;
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&Kd), sizeof(double) * KW * KW, s));
  k_float_to_double<<<(KW * KW + 255) / 256, 256, 0, s>>>(K, Kd, KW * KW);
  SRK_TRY(spectrum_from_spatial(Kd, KW, M, 1.0, nullptr, static_cast<float2*>(freq), s));
  SRK_CUDA(cudaFreeAsync(Kd, s));
  return SRK_OK;
}

srk_status srk_training_forward(const float* E, const float* I, const void* gx, const void* gy, int N, int W,
                                int erosion, float dx, int B, srk_stream_t s, float* R, srk_plan p) {
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_TRY(check_batch(p, B));
  SRK_NONNULL(E);
  SRK_NONNULL(I);
  SRK_NONNULL(R);
  if (p->spectra_M != N && (gx || gy))
    return fail(SRK_ERR_INVALID_ARG, "training spectra must be at size N=%d (plan has spectra_M=%d)", N, p->spectra_M);
  SRK_TRY(enter(p));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  OpArgs a = base_args(p);
  a.E = E; a.I = I; a.out0 = R;
  return launch_conv<OP_FWD, float>(p, a, fwd_geom(p, B), false, s);
}

srk_status srk_training_forward_sync(const float* E, const float* I, const void* gx, const void* gy, int N, int W,
                                     int erosion, float dx, int B, srk_stream_t s, float* R, srk_plan p) {
  SRK_TRY(srk_training_forward(E, I, gx, gy, N, W, erosion, dx, B, s, R, p));
  return srk_plan_sync(p, s);
}

srk_status srk_forward_oas(const float* E, const float* I, const void* gx, const void* gy, int N, int W,
                           int erosion, float dx, srk_stream_t s, float* R, srk_plan p, float* ux, float* uy) {
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_NONNULL(E);
  SRK_NONNULL(I);
  SRK_NONNULL(R);
  SRK_TRY(enter(p));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  OpArgs a = base_args(p);
  a.E = E; a.I = I; a.out0 = R; a.out_ux = ux; a.out_uy = uy;
  return launch_conv<OP_FWD, float>(p, a, fwd_geom(p, 1), false, s);
}

srk_status srk_adjoint(const float* v, const float* ux, const float* uy, const float* I, const void* gx,
                       const void* gy, int N, int W, int erosion, float dx, srk_stream_t s, float* dLdI, float* dLdE,
                       srk_plan p) {
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_NONNULL(v);
  SRK_NONNULL(ux);
  SRK_NONNULL(uy);
  SRK_NONNULL(I);
  SRK_NONNULL(dLdI);
  SRK_NONNULL(dLdE);
  SRK_TRY(enter(p));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  SRK_TRY(adj_wrt_f(p, nullptr, nullptr, v, ux, uy, 1, dLdI, s));
  return run_adj_g(p, v, nullptr, I, nullptr, 1, p->conv == SRK_ADJ_TRUE, dLdE, s);
}

srk_status srk_tangent(const float* f, const float* g, const float* df, const float* dg, const void* gx,
                       const void* gy, int N, int W, int erosion, float dx, srk_stream_t s, float* dh, srk_plan p) {
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(dh);
  SRK_TRY(enter(p));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.I = f; a.dI = df; a.out0 = dh;
  return launch_conv<OP_JVP, float>(p, a, fwd_geom(p, 1), false, s);
}

srk_status srk_tangent_adjoint(const float* f, const float* g, const float* df, const float* dg, const float* lam,
                               const float* dlam, const void* gx, const void* gy, int N, int W, int erosion, float dx,
                               srk_stream_t s, float* dLam_f, float* dLam_g, srk_plan p) {
  SRK_TRY(check_dims(p, N, W, erosion, dx));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(lam);
  SRK_NONNULL(dlam);
  SRK_NONNULL(dLam_f);
  SRK_NONNULL(dLam_g);
  SRK_TRY(enter(p));
  SRK_TRY(bind_spectra(p, gx, gy, s));
  const size_t ww = (size_t)p->W * p->W;
  SRK_TRY(ensure_wbuf(p, 2 * ww * sizeof(float), s));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.v = lam; a.dv = dlam; a.out0 = p->wbuf; a.out1 = p->wbuf + ww;
  SRK_TRY((launch_conv<OP_TANADJ_F, float>(p, a, fwd_geom(p, 1), false, s)));
  SRK_TRY(adj_wrt_f(p, p->wbuf, p->wbuf + ww, nullptr, nullptr, nullptr, 1, dLam_f, s));
  return run_adj_g(p, lam, dlam, f, df, 1, p->conv == SRK_ADJ_TRUE, dLam_g, s);
}

srk_status srk_forward(const float* f, const float* g, int B, srk_stream_t s, float* h, srk_plan p) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_TRY(check_batch(p, B));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(h);
  if (!p->have_G) return fail(SRK_ERR_INVALID_ARG, "no kernel set on the plan");
  SRK_TRY(enter(p));
  OpArgs a = base_args(p);
  a.E = g; a.I = f; a.out0 = h;
  return launch_conv<OP_FWD, float>(p, a, fwd_geom(p, B), false, s);
}

srk_status srk_vjp(const float* v, const float* f, const float* g, int B, srk_stream_t s, float* dLdf, float* dLdg,
                   srk_plan p) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_TRY(check_batch(p, B));
  SRK_NONNULL(v);
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(dLdf);
  SRK_NONNULL(dLdg);
  if (!p->have_G) return fail(SRK_ERR_INVALID_ARG, "no kernel set on the plan");
  SRK_TRY(enter(p));
  const size_t ww = (size_t)p->W * p->W * B;
  SRK_TRY(ensure_wbuf(p, 2 * ww * sizeof(float), s));
  OpArgs a = base_args(p);
  a.E = g; a.v = v; a.out0 = p->wbuf; a.out1 = p->wbuf + ww;
  SRK_TRY((launch_conv<OP_VJP_F, float>(p, a, fwd_geom(p, B), false, s)));
  // k_adj_wrt_f expects per-image wx, wy planes: [B][W][W] each
  SRK_TRY(adj_wrt_f(p, p->wbuf, p->wbuf + ww, nullptr, nullptr, nullptr, B, dLdf, s));
  return run_adj_g(p, v, nullptr, f, nullptr, B, true, dLdg, s);
}

srk_status srk_jvp(const float* f, const float* g, const float* df, const float* dg, int B, srk_stream_t s,
                   float* dh, srk_plan p) {
  if (!p) return fail(SRK_ERR_INVALID_ARG, "plan is NULL");
  SRK_TRY(check_batch(p, B));
  SRK_NONNULL(f);
  SRK_NONNULL(g);
  SRK_NONNULL(df);
  SRK_NONNULL(dg);
  SRK_NONNULL(dh);
  if (!p->have_G) return fail(SRK_ERR_INVALID_ARG, "no kernel set on the plan");
  SRK_TRY(enter(p));
  OpArgs a = base_args(p);
  a.E = g; a.dE = dg; a.I = f; a.dI = df; a.out0 = dh;
  return launch_conv<OP_JVP, float>(p, a, fwd_geom(p, B), false, s);
}

}  // extern "C"
