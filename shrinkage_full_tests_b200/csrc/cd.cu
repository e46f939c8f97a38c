// cd.cu — critical-dimension (CD) measurement of line/space signals, fused
// after the shrinkage operator.
//
// Algorithm (as MeasureCD_Batched, third_party/src/metricUtil/cd_measure_util.cu:310-437):
//   1. polyphase windowed-sinc table h[r][n], r < L, n in [-A, A]:
//        h = sinc(n - r/L) * Blackman((t + A) / 2A), t = n - r/L, each row
//        normalised to sum 1 (:56-82, :275-287);
//   2. L-fold upsampling up[m] = sum_n sig[k + n] h[r][n], m = k*L + r (:91-125);
//   3. zero crossings between up[i] and up[i+1] with linear sub-sample
//      position x = i - up[i]/(up[i+1]-up[i]) (:134-164);
//   4. nearest crossing left of the centre (N*L-1)/2 and nearest at or right
//      of it (:200-244); cd = (right - left) / L in input pixels (:254-266).
// Here one CTA does all four steps for one signal in shared memory: no
// intermediate buffers, no per-signal host loop, no host synchronisation.
// The table uses sinpi/cospi (the reference uses the __sinf/__cosf
// approximations; the difference is ~1e-6 of a tap).
#include "internal.h"

namespace srk {

constexpr int kCdThreads = 256;
constexpr int kCdMaxLen = 8192;  // samples per signal
constexpr int kCdMaxTaps = 1024; // L * (2A+1)

__device__ __forceinline__ float sinc_blackman_tap(float t, int A) {
  if (fabsf(t) > (float)A + 1e-6f) return 0.f;
  const float s = (fabsf(t) < 1e-6f) ? 1.f : sinpif(t) / (3.14159265358979f * t);
  const float u = (t + (float)A) / (float)(2 * A);
  const float bw = 0.42f - 0.5f * cospif(2.f * u) + 0.08f * cospif(4.f * u);
  return s * bw;
}

// Signal source: either explicit signals [B][n] (src == 0), or the centre
// line of E_crop + c*R built on the fly (src == 1: centre row, i.e. the
// line oy = W/2 along the columns; src == 2: centre column ox = W/2), as
// crop_center / apply_shrinkage / extract_center_row/col
// (training/main_cd_training.cu:126-165).
struct CdArgs {
  const float* sig;  // [B][n] (src 0)
  const float* E;    // [B][N][N] (src 1, 2)
  const float* R;    // [B][W][W] (src 1, 2)
  float coeff;
  int N, W, e, src;
};

__global__ void __launch_bounds__(kCdThreads) k_measure_cd(CdArgs a, int n, int L, int A, float* __restrict__ left_px,
                                                          float* __restrict__ right_px, float* __restrict__ cd_px) {
  __shared__ float s_sig[kCdMaxLen];
  __shared__ float s_h[kCdMaxTaps];
  __shared__ float s_red[2][kCdThreads / 32];
  const int b = blockIdx.x;
  const int taps = 2 * A + 1;
  // signal
  for (int j = threadIdx.x; j < n; j += kCdThreads) {
    float v;
    if (a.src == 0) {
      v = a.sig[(size_t)b * n + j];
    } else {
      const int W = a.W, N = a.N, e = a.e;
      const int ox = a.src == 1 ? j : W / 2;
      const int oy = a.src == 1 ? W / 2 : j;
      const float ec = a.E[(size_t)b * N * N + (size_t)(ox + e) * N + oy + e];
      v = ec + a.coeff * a.R[(size_t)b * W * W + (size_t)ox * W + oy];
    }
    s_sig[j] = v;
  }
  // polyphase table, one row per phase, normalised
  for (int r = threadIdx.x; r < L; r += kCdThreads) {
    const float phase = (float)r / (float)L;
    float sum = 0.f;
    for (int k = -A; k <= A; ++k) {
      const float w = sinc_blackman_tap((float)k - phase, A);
      s_h[r * taps + k + A] = w;
      sum += w;
    }
    const float inv = (fabsf(sum) > 1e-20f) ? 1.f / sum : 1.f;
    for (int i = 0; i < taps; ++i) s_h[r * taps + i] *= inv;
  }
  __syncthreads();
  auto up = [&](int m) {
    const int r = m % L, k = m / L;
    float acc = 0.f;
    for (int i = 0; i < taps; ++i) {
      const int idx = k + i - A;
      if ((unsigned)idx < (unsigned)n) acc += s_sig[idx] * s_h[r * taps + i];
    }
    return acc;
  };
  const int nup = n * L;
  const float centre = 0.5f * (float)(nup - 1);
  float best_l = -3.402823466e+38f, best_r = 3.402823466e+38f;
  for (int i = threadIdx.x; i < nup - 1; i += kCdThreads) {
    const float y0 = up(i), y1 = up(i + 1);
    if ((y0 <= 0.f && y1 > 0.f) || (y0 > 0.f && y1 <= 0.f)) {
      const float den = y1 - y0;
      const float x = (fabsf(den) < 1e-30f) ? (float)i : (float)i - y0 / den;
      if (x < centre) best_l = fmaxf(best_l, x);
      else best_r = fminf(best_r, x);
    }
  }
  // block reduction: max of left candidates, min of right candidates
  for (int o = 16; o > 0; o >>= 1) {
    best_l = fmaxf(best_l, __shfl_xor_sync(0xffffffffu, best_l, o));
    best_r = fminf(best_r, __shfl_xor_sync(0xffffffffu, best_r, o));
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { s_red[0][warp] = best_l; s_red[1][warp] = best_r; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float l = s_red[0][0], r = s_red[1][0];
    for (int w = 1; w < kCdThreads / 32; ++w) { l = fmaxf(l, s_red[0][w]); r = fminf(r, s_red[1][w]); }
    const float invL = 1.f / (float)L;
    left_px[b] = l * invL;
    right_px[b] = r * invL;
    cd_px[b] = (r - l) * invL;
  }
}

}  // namespace srk

using namespace srk;

extern "C" {

srk_status srk_measure_cd(const float* d_sig, int B, int n, int L, int A, srk_stream_t s, float* d_left,
                          float* d_right, float* d_cd) {
  if (!d_sig || !d_left || !d_right || !d_cd) return fail(SRK_ERR_INVALID_ARG, "NULL pointer");
  if (B < 1 || n < 2 || n > kCdMaxLen || L < 1 || A < 1 || L * (2 * A + 1) > kCdMaxTaps)
    return fail(SRK_ERR_INVALID_ARG, "need B>=1, 2<=n<=%d, L>=1, A>=1, L*(2A+1)<=%d (B=%d n=%d L=%d A=%d)", kCdMaxLen,
                kCdMaxTaps, B, n, L, A);
  CdArgs a{};
  a.sig = d_sig;
  a.src = 0;
  k_measure_cd<<<B, kCdThreads, 0, s>>>(a, n, L, A, d_left, d_right, d_cd);
  return cuda_status(cudaGetLastError(), "measure_cd launch");
}

srk_status srk_cd_after_shrinkage(const float* d_E, const float* d_R, int B, int N, int W, int erosion, float coeff,
                                  int axis, int L, int A, srk_stream_t s, float* d_left, float* d_right,
                                  float* d_cd) {
  if (!d_E || !d_R || !d_left || !d_right || !d_cd) return fail(SRK_ERR_INVALID_ARG, "NULL pointer");
  if (N < 3 || erosion < 0 || W != N - 2 * erosion || W < 2 || B < 1)
    return fail(SRK_ERR_INVALID_ARG, "bad sizes (N=%d W=%d erosion=%d B=%d)", N, W, erosion, B);
  if (axis != 0 && axis != 1) return fail(SRK_ERR_INVALID_ARG, "axis must be 0 (centre row) or 1 (centre column)");
  if (W > kCdMaxLen || L < 1 || A < 1 || L * (2 * A + 1) > kCdMaxTaps)
    return fail(SRK_ERR_INVALID_ARG, "W=%d, L=%d, A=%d out of range", W, L, A);
  CdArgs a{};
  a.E = d_E;
  a.R = d_R;
  a.coeff = coeff;
  a.N = N;
  a.W = W;
  a.e = erosion;
  a.src = axis == 0 ? 1 : 2;
  k_measure_cd<<<B, kCdThreads, 0, s>>>(a, W, L, A, d_left, d_right, d_cd);
  return cuda_status(cudaGetLastError(), "cd launch");
}

}  // extern "C"
