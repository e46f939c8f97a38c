// hybrid_p1.cuh — the column pass (P1) of the tensor-core row schedule
// (SRK_SCHEDULE_TENSOR_ROWS): the same column FFT along y as the engine's P1
// at M = 512, but its output is written as FP16 planes, one per (ky, part),
// in the layout the tensor-core row pass (hybrid.cu) reads with TMA:
//   planes[((ky * 2 + part) * c + wl) * M + x]      (part 0 = re, 1 = im),
// c = work tiles in the chunk, wl = work tile within the chunk.  Each CTA
// transforms 8 consecutive columns (two units of four), stages their values
// [ky][part][8] in shared memory and writes them with TMA stores (one
// 16-byte piece per (ky, part) plane row).  Used for the pair ops (OP_FWD,
// OP_VJP_F: two images per work tile) where the column DFT of
// hybrid_p1g.cuh does not apply, and by the refit pass.
#pragma once
#include <cuda.h>

#include "engine.cuh"
#include "hybrid_scale.cuh"
#include "tc.cuh"

namespace srk {

constexpr int kHybM = 512;

// Shared memory of k_p1h / k_p1h_refit, all dynamic (static __shared__
// variables would move the dynamic block off the 128-byte boundary the TMA
// stores need): the engine's phase layout, the FP16 staging block
// [M][2][kP1hCols], then the refit's work list (P1hAux).
// 8 columns per CTA (16 bytes per (ky, part)): measured 0.66 ms per 500 work
// tiles against 0.81 ms with 16 columns (whole 32-byte sectors, but 3 CTAs
// per SM and twice the transforms per line).
constexpr int kP1hCols = 8;
// Byte offset of the staging block (128-byte aligned: the source of TMA stores).
__host__ __device__ constexpr size_t p1h_stage_offset() { return (phase_smem_bytes<kHybM>() + 127) / 128 * 128; }
struct P1hAux {
  int cnt[kWarps];     // refit: flagged work tiles per warp
  int list[kThreads];  // refit: the flagged work tiles of one group
};
__host__ __device__ constexpr size_t p1h_aux_offset() {
  return p1h_stage_offset() + (size_t)kHybM * 2 * kP1hCols * sizeof(__half);
}
__host__ __device__ constexpr size_t p1h_smem_bytes() { return p1h_aux_offset() + sizeof(P1hAux); }
// Planes written per TMA store (box {8 columns, 1 work tile, kP1hBox planes}).
constexpr int kP1hBox = 256;

// The column pass of the kP1hCols columns kP1hCols * xb .. of work tile wl
// (w = w0 + wl): FFTs along y, values times sp rounded to FP16 and staged
// [plane = 2 ky + part][8 columns], written by TMA stores (box {8 columns, 1
// work tile, kP1hBox planes}: the TMA engine writes the 1024 16-byte row
// pieces the threads would otherwise scatter).  Block-uniform arguments; the
// twiddles are in sm.  With zmax given, each warp folds the max |Z| of its
// unscaled values into zmax[wl] (one atomic per warp, float bits).  Ends with
// the stores complete and the block synchronised (the staging block may be
// reused).
template <int OP, typename T>
__device__ __forceinline__ void p1h_cols(const CUtensorMap* pmap, const OpArgs& a, const Geom& g, float2* sm,
                                         int w0, int wl, int xb, float sp, int ahead, unsigned int* zmax,
                                         unsigned int* err) {
  constexpr int M = kHybM;
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  constexpr int LPU = lpu_of<M>();
  constexpr int NU = kP1hCols / LPU;  // units of LPU columns per CTA
  const int line = threadIdx.x / TPF, t = threadIdx.x % TPF;
  float2* rows = sm + tw_slots<M>();
  __half* st = reinterpret_cast<__half*>(reinterpret_cast<unsigned char*>(sm) + p1h_stage_offset());
  const int w = w0 + wl;
  if (ahead > 0) {
    // L2 prefetch of the image columns of the CTA one SM-count of launch positions later
    const int lin = (int)(blockIdx.y * gridDim.x + blockIdx.x) + ahead;
    const int w2 = w - (int)blockIdx.y + lin / (int)gridDim.x, xb2 = (lin % (int)gridDim.x) * NU;
    for (int u = 0; u < NU; u += 2) p1_prefetch<M, OP, T, 2>(a, g, w2, xb2 + u);
  }
  float2* row = rows + line * row_stride<M>();
  float2 za[EPT], zb[EPT];
  float m = 0.f;
  load_column<M, OP, T>(a, g, w, 0, (NU * xb) * LPU + line, t, za);
#pragma unroll 1
  for (int u = 0; u < NU; ++u) {
    // the next unit's column loads are in flight during this transform
    if (u + 1 < NU) load_column<M, OP, T>(a, g, w, 0, (NU * xb + u + 1) * LPU + line, t, zb);
    fft<M, false>(za, row, sm, t, 1 + line);
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int ky = t + TPF * i;
      m = fmaxf(m, fmaxf(fabsf(za[i].x), fabsf(za[i].y)));
      st[(ky * 2 + 0) * kP1hCols + u * LPU + line] = __float2half_rn(za[i].x * sp);
      st[(ky * 2 + 1) * kP1hCols + u * LPU + line] = __float2half_rn(za[i].y * sp);
    }
#pragma unroll
    for (int i = 0; i < EPT; ++i) za[i] = zb[i];
  }
  if (zmax) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(zmax + wl, __float_as_uint(m));
  }
  tc::fence_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    if ((tc::smem_u32(st) & 127u) == 0) {
      for (int p0 = 0; p0 < 2 * M; p0 += kP1hBox) tc::tma_store_3d(pmap, xb * kP1hCols, wl, p0, st + p0 * kP1hCols);
      tc::bulk_commit();
    } else {
      atomicCAS(err, 0u, 15u);  // the TMA source must sit on 128 bytes: record, store nothing
    }
    tc::bulk_wait_all();
  }
  __syncthreads();
}

// First column pass of a chunk: every work tile's planes at scale 1, and
// zmax[wl] = max |Z| of work tile wl (float bits; zeroed before the launch).
// Grid (M / kP1hCols, c).
template <int OP, typename T>
__global__ void __launch_bounds__(kThreads, SRK_P1_MIN_BLOCKS)
k_p1h(const __grid_constant__ CUtensorMap pmap, OpArgs a, Geom g, const float2* __restrict__ twg, int w0, int ahead,
      unsigned int* __restrict__ zmax, unsigned int* err) {
  static_assert(OpTraits<OP>::K == 1, "single-field ops only");
  extern __shared__ __align__(128) float2 sm[];
  load_twiddles(sm, twg, kHybM);
  __syncthreads();
  p1h_cols<OP, T>(&pmap, a, g, sm, w0, blockIdx.y, blockIdx.x, 1.f, ahead, zmax, err);
}

// Refit: the work tiles whose zmax lies outside the range kept at scale 1
// (plane_exp != 0) are transformed again, their planes written at scale
// 2^plane_exp.  Persistent over the (work tile, column block) units of the
// flagged work tiles, in order; every block scans zmax (c words) for them, so
// a chunk without such work tiles costs one short launch.
template <int OP, typename T>
__global__ void __launch_bounds__(kThreads, SRK_P1_MIN_BLOCKS)
k_p1h_refit(const __grid_constant__ CUtensorMap pmap, OpArgs a, Geom g, const float2* __restrict__ twg, int w0, int c,
            const unsigned int* __restrict__ zmax, unsigned int* err) {
  constexpr int NX = kHybM / kP1hCols;  // column blocks per work tile
  extern __shared__ __align__(128) float2 sm[];
  P1hAux* aux = reinterpret_cast<P1hAux*>(reinterpret_cast<unsigned char*>(sm) + p1h_aux_offset());
  int* cnt = aux->cnt;
  int* list = aux->list;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool loaded = false;
  long long rank0 = 0;  // flagged work tiles before this group of kThreads
  for (int b0 = 0; b0 < c; b0 += kThreads) {
    const int wl = b0 + threadIdx.x;
    const bool f = wl < c && plane_exp(__ldg(zmax + wl)) != 0;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) cnt[warp] = __popc(bal);
    __syncthreads();
    int before = 0, total = 0;
    for (int i = 0; i < kWarps; ++i) {
      before += i < warp ? cnt[i] : 0;
      total += cnt[i];
    }
    if (f) list[before + __popc(bal & ((1u << lane) - 1u))] = wl;
    __syncthreads();
    for (int k = 0; k < total; ++k) {
      const int wk = list[k];
      const float sp = ldexpf(1.f, plane_exp(__ldg(zmax + wk)));
      for (int xb = 0; xb < NX; ++xb) {
        if ((int)(((rank0 + k) * NX + xb) % gridDim.x) != (int)blockIdx.x) continue;
        if (!loaded) {
          load_twiddles(sm, twg, kHybM);
          __syncthreads();
          loaded = true;
        }
        p1h_cols<OP, T>(&pmap, a, g, sm, w0, wk, xb, sp, 0, nullptr, err);
      }
    }
    rank0 += total;
    __syncthreads();  // cnt and list are rewritten by the next group
  }
}

}  // namespace srk
