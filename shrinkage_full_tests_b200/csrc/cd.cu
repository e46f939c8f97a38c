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

// ---- CD of the shrunk pattern without the full operator ------------------------
// When only the CD is wanted, R is needed on one line per image: the centre
// row (axis 0: oy = W/2, ox = 0..W-1) or column (axis 1).  k_strip_line
// computes ux, uy there by direct convolution (the strip idea of
// training/main_compare.cu:70-133, which uses cuDNN on a KW-row strip), then
// the signal E + c*R on that line (crop_center / apply_shrinkage,
// training/main_cd_training.cu:126-165).  Line positions p (x for axis 0,
// y for axis 1), band positions q (the other axis, KW of them).
// CTA: 256 consecutive outputs of one image; lane l owns outputs 8l .. 8l+7,
// warp w the band lines q = w, w+8, ... of each 32-line chunk, staged in
// shared memory (padding p + p/8 keeps the lanes' stride-8 reads on distinct
// banks).  Taps come from Kt[q][s] (s = c - line offset, zero past KW, 8-
// aligned rows), read warp-uniformly.
constexpr int kStripOut = 256;
constexpr int kStripQC = 32;  // band lines per staged chunk

__global__ void k_strip_taps(const float* __restrict__ Kx, const float* __restrict__ Ky, int KW, int KW8, int axis,
                             float* __restrict__ Ktx, float* __restrict__ Kty) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= KW * KW8) return;
  const int q = i / KW8, sidx = i - (i / KW8) * KW8;
  const int c = KW / 2;
  float vx = 0.f, vy = 0.f;
  if (sidx < KW) {
    const int k = axis == 0 ? (2 * c - sidx) * KW + (2 * c - q) : (2 * c - q) * KW + (2 * c - sidx);
    vx = Kx[k];
    vy = Ky[k];
  }
  Ktx[i] = vx;
  Kty[i] = vy;
}

__device__ __forceinline__ int strip_pad(int p) { return p + (p >> 3); }

__global__ void __launch_bounds__(256, 2)
k_strip_line(const float* __restrict__ E, const float* __restrict__ I, const float* __restrict__ Ktx,
             const float* __restrict__ Kty, int KW, int KW8, int N, int W, int e, float dx2, float coeff, int axis,
             float* __restrict__ sig) {
  extern __shared__ float strip_sm[];
  float* sm = strip_sm;
  const int c = KW / 2;
  const int TP = kStripOut + KW8;                 // staged line positions (>= 256 + 2c + 8)
  const int TPP = strip_pad(TP) | 1;              // odd pitch: conflict-free staging stores
  const int b = blockIdx.y, p0 = blockIdx.x * kStripOut;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float* img = E + (long long)b * N * N;
  const int line_img = W / 2 + e;                 // image coordinate of the line on the band axis
  const int pstart = p0 + e - c;                  // image coordinate of staged line position 0
  float ux[8], uy[8];
#pragma unroll
  for (int m = 0; m < 8; ++m) ux[m] = uy[m] = 0.f;
  for (int qc0 = 0; qc0 < KW; qc0 += kStripQC) {
    const int nq = min(kStripQC, KW - qc0);
    __syncthreads();  // the previous chunk is consumed
    for (int idx = threadIdx.x; idx < nq * TP; idx += 256) {
      int qq, pl;
      if (axis == 0) { qq = idx % nq; pl = idx / nq; } else { pl = idx % TP; qq = idx / TP; }
      const int pimg = pstart + pl;                       // line coordinate
      const int qimg = line_img - c + qc0 + qq;           // band coordinate
      float v = 0.f;
      if (pimg < N) v = axis == 0 ? img[(long long)pimg * N + qimg] : img[(long long)qimg * N + pimg];
      sm[qq * TPP + strip_pad(pl)] = v;
    }
    __syncthreads();
    for (int qq = warp; qq < nq; qq += 8) {
      const float* row = sm + qq * TPP;
      const float* kx = Ktx + (long long)(qc0 + qq) * KW8;
      const float* ky = Kty + (long long)(qc0 + qq) * KW8;
      float v[16];
#pragma unroll
      for (int j = 0; j < 8; ++j) v[8 + j] = row[strip_pad(8 * lane + j)];
      for (int s0 = 0; s0 < KW8; s0 += 8) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          v[j] = v[8 + j];
          v[8 + j] = row[strip_pad(8 * lane + s0 + 8 + j)];
        }
        // 8 taps of each kernel as two 16-byte loads (rows are 8-aligned)
        const float4 ax = __ldg(reinterpret_cast<const float4*>(kx + s0));
        const float4 bx = __ldg(reinterpret_cast<const float4*>(kx + s0) + 1);
        const float4 ay = __ldg(reinterpret_cast<const float4*>(ky + s0));
        const float4 by = __ldg(reinterpret_cast<const float4*>(ky + s0) + 1);
        const float wxs[8] = {ax.x, ax.y, ax.z, ax.w, bx.x, bx.y, bx.z, bx.w};
        const float wys[8] = {ay.x, ay.y, ay.z, ay.w, by.x, by.y, by.z, by.w};
#pragma unroll
        for (int st = 0; st < 8; ++st) {
#pragma unroll
          for (int m = 0; m < 8; ++m) {
            ux[m] = __fmaf_rn(wxs[st], v[m + st], ux[m]);
            uy[m] = __fmaf_rn(wys[st], v[m + st], uy[m]);
          }
        }
      }
    }
  }
  // reduce the 8 warps' partial sums, then the signal E + c*R on the line
  __syncthreads();
  float* red = sm;  // [8 warps][256 outputs][2]
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    red[(warp * kStripOut + 8 * lane + m) * 2] = ux[m];
    red[(warp * kStripOut + 8 * lane + m) * 2 + 1] = uy[m];
  }
  __syncthreads();
  const int o = p0 + threadIdx.x;
  if (o >= W) return;
  float sx = 0.f, sy = 0.f;
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    sx += red[(w * kStripOut + threadIdx.x) * 2];
    sy += red[(w * kStripOut + threadIdx.x) * 2 + 1];
  }
  const int gx = axis == 0 ? o + e : line_img, gy = axis == 0 ? line_img : o + e;
  const float* fi = I + (long long)b * N * N;
  // central differences (erosion >= 1: the neighbours are inside the image)
  const float fx = (fi[(long long)(gx + 1) * N + gy] - fi[(long long)(gx - 1) * N + gy]) * 0.5f;
  const float fy = (fi[(long long)gx * N + gy + 1] - fi[(long long)gx * N + gy - 1]) * 0.5f;
  const float R = __fmaf_rn(dx2 * sx, fx, __fmul_rn(dx2 * sy, fy));
  sig[(long long)b * W + o] = img[(long long)gx * N + gy] + coeff * R;
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

srk_status srk_cd_strip(const float* d_E, const float* d_I, const float* d_Kx, const float* d_Ky, int KW, int N,
                        int W, int erosion, float dx, int B, float coeff, int axis, int L, int A, srk_stream_t s,
                        float* d_left, float* d_right, float* d_cd) {
  if (!d_E || !d_I || !d_Kx || !d_Ky || !d_left || !d_right || !d_cd) return fail(SRK_ERR_INVALID_ARG, "NULL pointer");
  if (N < 3 || erosion < 1 || W != N - 2 * erosion || W < 2 || B < 1 || B > 65535)
    return fail(SRK_ERR_INVALID_ARG, "bad sizes (N=%d W=%d erosion=%d B=%d)", N, W, erosion, B);
  if (KW < 1 || !(KW & 1) || KW > 2 * erosion + 1 || KW > 129)
    return fail(SRK_ERR_INVALID_ARG, "KW=%d must be odd, <= 2*erosion+1 and <= 129", KW);
  if (axis != 0 && axis != 1) return fail(SRK_ERR_INVALID_ARG, "axis must be 0 (centre row) or 1 (centre column)");
  if (W > kCdMaxLen || L < 1 || A < 1 || L * (2 * A + 1) > kCdMaxTaps)
    return fail(SRK_ERR_INVALID_ARG, "W=%d, L=%d, A=%d out of range", W, L, A);
  if (!(dx > 0.f)) return fail(SRK_ERR_INVALID_ARG, "dx=%g must be positive", dx);
  const int KW8 = (KW + 7) & ~7;
  const int TP = kStripOut + KW8;
  const int TPP = (TP + (TP >> 3)) | 1;
  const size_t smem = sizeof(float) * std::max<size_t>((size_t)kStripQC * TPP, (size_t)8 * kStripOut * 2);
  SRK_CUDA(cudaFuncSetAttribute(k_strip_line, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  float* buf = nullptr;
  const size_t nt = (size_t)KW * KW8;
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&buf), sizeof(float) * (2 * nt + (size_t)B * W), s));
  float* ktx = buf;
  float* kty = buf + nt;
  float* sig = buf + 2 * nt;
  k_strip_taps<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(d_Kx, d_Ky, KW, KW8, axis, ktx, kty);
  k_strip_line<<<dim3((W + kStripOut - 1) / kStripOut, B), 256, smem, s>>>(d_E, d_I, ktx, kty, KW, KW8, N, W, erosion,
                                                                           dx * dx, coeff, axis, sig);
  CdArgs a{};
  a.sig = sig;
  a.src = 0;
  k_measure_cd<<<B, kCdThreads, 0, s>>>(a, W, L, A, d_left, d_right, d_cd);
  SRK_CUDA(cudaGetLastError());
  SRK_CUDA(cudaFreeAsync(buf, s));
  return SRK_OK;
}

}  // extern "C"
