// hybrid_p1.cuh — the column pass (P1) of the tensor-core row schedule
// (SRK_SCHEDULE_TENSOR_ROWS): the same column FFT along y as the engine's P1
// at M = 512, but its output is written as FP16 planes, one per (ky, part),
// in the layout the tensor-core row pass (hybrid.cu) reads with TMA:
//   planes[((ky * 2 + part) * c + wl) * M + x]      (part 0 = re, 1 = im),
// c = work tiles in the chunk, wl = work tile within the chunk.  Each CTA
// transforms 8 consecutive columns (two units of four), stages their values
// [ky][part][8] in shared memory and writes them with TMA stores (one
// 16-byte piece per (ky, part) plane row).  Only for single-field
// ops (one complex field per work tile: OP_FWD, OP_VJP_F, OP_JVP,
// OP_TANADJ_F).
#pragma once
#include <cuda.h>

#include "engine.cuh"
#include "tc.cuh"

namespace srk {

constexpr int kHybM = 512;

// Shared memory of k_p1h: the engine's phase layout plus the FP16 staging
// block [M][2][kP1hCols].  8 columns per CTA (16 bytes per (ky, part)):
// measured 0.66 ms per 500 work tiles against 0.81 ms with 16 columns
// (whole 32-byte sectors, but 3 CTAs per SM and twice the transforms per
// line).
constexpr int kP1hCols = 8;
// Byte offset of the staging block (128-byte aligned: the source of TMA stores).
__host__ __device__ constexpr size_t p1h_stage_offset() { return (phase_smem_bytes<kHybM>() + 127) / 128 * 128; }
__host__ __device__ constexpr size_t p1h_smem_bytes() {
  return p1h_stage_offset() + (size_t)kHybM * 2 * kP1hCols * sizeof(__half);
}
// Planes written per TMA store (box {8 columns, 1 work tile, kP1hBox planes}).
constexpr int kP1hBox = 256;

template <int OP, typename T>
__global__ void __launch_bounds__(kThreads, SRK_P1_MIN_BLOCKS)
k_p1h(const __grid_constant__ CUtensorMap pmap, OpArgs a, Geom g, const float2* __restrict__ twg, int w0, int ahead) {
  constexpr int M = kHybM;
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  constexpr int LPU = lpu_of<M>();
  constexpr int NU = kP1hCols / LPU;  // units of LPU columns per CTA
  static_assert(OpTraits<OP>::K == 1, "single-field ops only");
  extern __shared__ float2 sm[];
  const int line = threadIdx.x / TPF, t = threadIdx.x % TPF;
  load_twiddles(sm, twg, M);
  __syncthreads();
  float2* rows = sm + tw_slots<M>();
  __half* st = reinterpret_cast<__half*>(reinterpret_cast<unsigned char*>(sm) + p1h_stage_offset());  // [ky][part][8]
  const int wl = blockIdx.y, w = w0 + wl;
  const int xb = blockIdx.x;  // columns kP1hCols * xb ..
  if (ahead > 0) {
    // L2 prefetch of the image columns of the CTA one SM-count of launch positions later
    const int lin = (int)(blockIdx.y * gridDim.x + blockIdx.x) + ahead;
    const int w2 = w - (int)blockIdx.y + lin / (int)gridDim.x, xb2 = (lin % (int)gridDim.x) * NU;
    for (int u = 0; u < NU; u += 2) p1_prefetch<M, OP, T, 2>(a, g, w2, xb2 + u);
  }
  float2* row = rows + line * row_stride<M>();
  float2 za[EPT], zb[EPT];
  load_column<M, OP, T>(a, g, w, 0, (NU * xb) * LPU + line, t, za);
#pragma unroll 1
  for (int u = 0; u < NU; ++u) {
    // the next unit's column loads are in flight during this transform
    if (u + 1 < NU) load_column<M, OP, T>(a, g, w, 0, (NU * xb + u + 1) * LPU + line, t, zb);
    fft<M, false>(za, row, sm, t, 1 + line);
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int ky = t + TPF * i;
      st[(ky * 2 + 0) * kP1hCols + u * LPU + line] = __float2half_rn(za[i].x);
      st[(ky * 2 + 1) * kP1hCols + u * LPU + line] = __float2half_rn(za[i].y);
    }
#pragma unroll
    for (int i = 0; i < EPT; ++i) za[i] = zb[i];
  }
  // the staging block [plane = 2 ky + part][8 columns] is the layout of the
  // store box {8 columns, 1 work tile, kP1hBox planes}: the TMA engine writes
  // the 1024 16-byte row pieces (the threads would need 1024 scattered stores)
  tc::fence_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int p0 = 0; p0 < 2 * M; p0 += kP1hBox) tc::tma_store_3d(&pmap, xb * kP1hCols, wl, p0, st + p0 * kP1hCols);
    tc::bulk_commit();
    tc::bulk_wait_all();
  }
}

}  // namespace srk
