// hybrid_p1.cuh — the column pass (P1) of the tensor-core row schedule
// (SRK_SCHEDULE_TENSOR_ROWS): the same column FFT along y as the engine's P1
// at M = 512, but its output is written as FP16 planes, one per (ky, part),
// in the layout the tensor-core row pass (hybrid.cu) reads with TMA:
//   planes[((ky * 2 + part) * c + wl) * M + x]      (part 0 = re, 1 = im),
// c = work tiles in the chunk, wl = work tile within the chunk.  Each CTA
// transforms 8 consecutive columns (two units of four) and writes, for every
// (ky, part), their 8 values as one 16-byte store.  Only for single-field
// ops (one complex field per work tile: OP_FWD, OP_VJP_F, OP_JVP,
// OP_TANADJ_F).
#pragma once
#include "engine.cuh"

namespace srk {

constexpr int kHybM = 512;

// Shared memory of k_p1h: the engine's phase layout plus the FP16 staging
// block [M][2][kP1hCols].  8 columns per CTA (16 bytes per (ky, part)):
// measured 0.66 ms per 500 work tiles against 0.81 ms with 16 columns
// (whole 32-byte sectors, but 3 CTAs per SM and twice the transforms per
// line).
constexpr int kP1hCols = 8;
__host__ __device__ constexpr size_t p1h_smem_bytes() {
  return phase_smem_bytes<kHybM>() + (size_t)kHybM * 2 * kP1hCols * sizeof(__half);
}

template <int OP, typename T>
__global__ void __launch_bounds__(kThreads, SRK_P1_MIN_BLOCKS)
k_p1h(OpArgs a, Geom g, const float2* __restrict__ twg, int w0, __half* __restrict__ planes, int c, int ahead) {
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
  __half* st = reinterpret_cast<__half*>(rows + 2 * LPU * row_stride<M>());  // [ky][part][kP1hCols columns]
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
  __syncthreads();
  const size_t x0 = (size_t)xb * kP1hCols;
  constexpr int PIECES = kP1hCols / 8;  // 16-byte pieces per (ky, part)
  for (int j = threadIdx.x; j < M * 2 * PIECES; j += kThreads) {
    const int plane = j / PIECES, piece = j % PIECES;
    __stcg(reinterpret_cast<uint4*>(planes + ((size_t)plane * c + wl) * M + x0 + 8 * piece),
           *reinterpret_cast<const uint4*>(st + plane * kP1hCols + 8 * piece));
  }
}

}  // namespace srk
