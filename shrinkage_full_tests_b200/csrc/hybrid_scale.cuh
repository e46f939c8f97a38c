// hybrid_scale.cuh — the per-work-tile power-of-two scale of the FP16 column
// spectra planes of SRK_SCHEDULE_TENSOR_ROWS, shared by the column pass that
// writes them (hybrid_p1.cuh) and the row pass that reads them (hybrid.cu).
#pragma once
#include <cuda_runtime.h>

namespace srk {

// S2 layout the row pass writes and P3 reads (S2Layout in engine.cuh):
// 1 = blocked with rotated lines, 2 = plain [field][ky][pitch].  Measured per
// 128 work tiles: rotated blocks 140 + 188 us (row pass + P3), plain 129 +
// 264 us (coalesced row-pass stores, 32-byte P3 reads).
#ifndef SRK_HYB_S2_LAYOUT
#define SRK_HYB_S2_LAYOUT 1
#endif
constexpr int kHybS2Layout = SRK_HYB_S2_LAYOUT;

// FP16 range of the planes.  A column spectrum value is a sum of M = 512
// complex inputs (|Z.x|, |Z.y| <= 2^10 max|input|) and FP16 holds at most
// 65504 with full precision only above 2^-14: unscaled, an FP16 or BF16
// image with values above 64 could overflow.  The planes of a work tile are
// written at scale 1 when its largest |Z| lies in [2^-8, kPlaneHi] — below
// 65504 with room for rounding, and high enough that the values in FP16's
// subnormal range (below 2^-14, absolute error <= 2^-25) err by less than
// 2^-17 of the largest — which holds for images of order 1e-4 .. 60, so
// typical inputs need no second pass.  Otherwise (k_p1h_refit) they are
// written at 2^p with
// p = 15 - q, largest |Z| = f 2^q, f in [0.5, 1): |Z 2^p| < 2^15.  The row
// pass multiplies each work tile's sums (one MMA column) by 2^-(p + t), t
// the band tables' exponent — a power of two, no rounding of its own.  p is
// kept in [-64, 64] (|t| <= 60), so that factor is a normal float: images
// of magnitude about 1e-22 .. 1e19 (FP16's range, and most of BF16's).
constexpr float kPlaneHi = 65000.f;
constexpr float kPlaneLo = 0.00390625f;  // 2^-8

// p for a work tile whose largest |Z| has the float bits zbits (0: scale 1).
__device__ __forceinline__ int plane_exp(unsigned int zbits) {
  const float z = __uint_as_float(zbits);
  if (!(z > kPlaneHi) && !(z > 0.f && z < kPlaneLo)) return 0;  // in range, all zero or NaN
  if (z > 3.0e38f) return -64;                                   // infinities propagate
  int q = 0;
  frexpf(z, &q);
  const int p = 15 - q;
  return p < -64 ? -64 : (p > 64 ? 64 : p);
}

}  // namespace srk
