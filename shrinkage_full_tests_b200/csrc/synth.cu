// synth.cu — synthetic inputs on the device: Gaussian random fields (GRF)
// and line/space (LNS) patterns, batched.
//
// GRF, as GpGenerator (third_party/include/stTestCore/gp_generator.h:95-254):
// white N(0,1) noise on the Np x Np grid (Np = next power of two >= N),
// filtered by H = sqrt(FFT2(c)) of the periodic covariance
// c(dx, dy) = exp(-(dx^2 + dy^2) / (2 ell^2)) (nearest-image displacements),
// cropped to the top-left N x N.  The covariance is separable, so the filter
// is the circular convolution with h(dx) h(dy), h = IFFT1(sqrt(FFT1(c1)))
// (1/Np normalised): two 1-D passes of 2R+1 taps here instead of two 2-D
// FFTs, R chosen so the dropped taps are below 1e-9 of h(0) (or the whole
// period, when that is shorter).  Optionally each
// image is min-max scaled to [0, 1] (the training inputs).
//
// Noise: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011) keyed by (seed + image), counter =
// pixel / 4, and the Box-Muller transform; one normal per pixel, image b
// independent of the batch it is generated in.
//
// LNS, as gen_lns_vertical / gen_lns_horizontal
// (third_party/src/patternUtil/test_pattern.cu:83-109, lns_value :71-80): a
// Gaussian pulse train of 2*nbrs+1 lines around the centre, minus 0.5.
#include "internal.h"

namespace srk {
namespace {

constexpr int kSynThreads = 256;
constexpr int kMaxTaps = 1025;  // 2R+1

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k.x += 0x9E3779B9u;
      k.y += 0xBB67AE85u;
    }
    const unsigned lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const unsigned lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
  }
  return c;
}

// Uniform in (0, 1): (bits + 0.5) / 2^32.
__device__ __forceinline__ float u01(unsigned b) { return ((float)b + 0.5f) * 2.3283064365386963e-10f; }

// Noise of `nb` images starting at image b0 (key seed + b), col-major Np x Np.
__global__ void k_grf_noise(float* __restrict__ w, int Np, unsigned long long seed, int b0) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // group of 4 pixels
  const long long npx = (long long)Np * Np;
  if (4 * q >= npx) return;
  const int b = blockIdx.y;
  const unsigned long long key = seed + (unsigned long long)(b0 + b);
  const uint4 r = philox4x32_10(make_uint4((unsigned)q, (unsigned)(q >> 32), 0u, 0u),
                                make_uint2((unsigned)key, (unsigned)(key >> 32)));
  float s0, c0, s1, c1;
  const float m0 = sqrtf(-2.f * logf(u01(r.x))), m1 = sqrtf(-2.f * logf(u01(r.z)));
  sincospif(2.f * u01(r.y), &s0, &c0);
  sincospif(2.f * u01(r.w), &s1, &c1);
  float4 v = make_float4(m0 * c0, m0 * s0, m1 * c1, m1 * s1);
  float* dst = w + (long long)b * npx + 4 * q;  // Np >= 4 and a power of two: 16-byte aligned
  *reinterpret_cast<float4*>(dst) = v;
}

// Pass along x (columns): t[x][y] = sum_d h(d) w[(x - d) mod Np][y], x < N,
// y < Np.  Block: 32 rows (lanes) x 64 columns (8 warps x 8 outputs).  The
// taps come zero-padded (hz[m - i + 7], see grf_taps) so every lane runs the
// same branch-free sliding window.
__global__ void k_grf_conv_x(const float* __restrict__ w, float* __restrict__ t, int Np, int N, int R,
                             const float* __restrict__ hz) {
  extern __shared__ float sm[];
  const int ntap = 2 * R + 15;
  float* taps = sm;
  float* tile = sm + ntap;  // [(64 + 2R) columns][32 rows]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int y0 = blockIdx.x * 32, x0 = blockIdx.y * 64, b = blockIdx.z;
  const float* src = w + (long long)b * Np * Np;
  for (int i = threadIdx.x; i < ntap; i += kSynThreads) taps[i] = hz[i];
  const int ncol = 64 + 2 * R;
  const bool row_ok = y0 + lane < Np;  // Np < 32 for small images
  for (int c = warp; c < ncol; c += 8) {
    const int x = ((x0 - R + c) % Np + Np) % Np;
    tile[c * 32 + lane] = row_ok ? src[(long long)x * Np + y0 + lane] : 0.f;
  }
  __syncthreads();
  float o[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) o[i] = 0.f;
  const float* col = tile + (8 * warp) * 32 + lane;
  for (int m = 0; m < 8 + 2 * R; ++m) {
    const float v = col[m * 32];
#pragma unroll
    for (int i = 0; i < 8; ++i) o[i] = __fmaf_rn(taps[m - i + 7], v, o[i]);
  }
  float* dst = t + (long long)b * N * Np;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int x = x0 + 8 * warp + i;
    if (x < N && row_ok) dst[(long long)x * Np + y0 + lane] = o[i];
  }
}

__device__ __forceinline__ unsigned order_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float order_val(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// Pass along y: out[x][y] (+)= sum_d h(d) t[x][(y - d) mod Np], x, y < N.
// Block: 8 columns (warps) x 256 rows (lane l: rows 8l .. 8l+7); the staged
// column uses the padding i + i/8 so the lanes' stride-8 window reads hit 32
// distinct banks.  Also the per-image min and max (order-preserving keys).
__global__ void k_grf_conv_y(const float* __restrict__ t, float* __restrict__ out, int Np, int N, int R,
                             const float* __restrict__ hz, unsigned* __restrict__ mm, int B, int accumulate) {
  extern __shared__ float sm[];
  const int ntap = 2 * R + 15;
  const int H = 256 + 2 * R;
  const int HP = H + H / 8 + 1;
  float* taps = sm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int y0 = blockIdx.x * 256, x = blockIdx.y * 8 + warp, b = blockIdx.z;
  float* col = sm + ntap + warp * HP;
  for (int i = threadIdx.x; i < ntap; i += kSynThreads) taps[i] = hz[i];
  const bool live = x < N;
  if (live) {
    const float* src = t + (long long)b * N * Np + (long long)x * Np;
    for (int r = lane; r < H; r += 32) {
      const int y = ((y0 - R + r) % Np + Np) % Np;
      col[r + (r >> 3)] = src[y];
    }
  }
  __syncthreads();
  float lo = 3.402823466e+38f, hi = -3.402823466e+38f;
  if (live) {
    float o[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) o[i] = 0.f;
    for (int m = 0; m < 8 + 2 * R; ++m) {
      const int idx = 8 * lane + m;
      const float v = col[idx + (idx >> 3)];
#pragma unroll
      for (int i = 0; i < 8; ++i) o[i] = __fmaf_rn(taps[m - i + 7], v, o[i]);
    }
    float* dst = out + (long long)b * N * N + (long long)x * N;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int y = y0 + 8 * lane + i;
      if (y < N) {
        const float v = accumulate ? __fadd_rn(dst[y], o[i]) : o[i];
        dst[y] = v;
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
      }
    }
  }
  if (mm) {
    for (int s = 16; s > 0; s >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, s));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, s));
    }
    if (lane == 0 && live) {
      atomicMin(mm + b, order_key(lo));
      atomicMax(mm + B + b, order_key(hi));
    }
  }
}

__global__ void k_minmax_scale(float* __restrict__ out, int N, const unsigned* __restrict__ mm, int B) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (i >= (long long)N * N) return;
  const float lo = order_val(mm[b]), hi = order_val(mm[B + b]);
  float* p = out + (long long)b * N * N + i;
  *p = hi > lo ? (*p - lo) / (hi - lo) : 0.f;
}

// Line/space: one value per column (vertical) or per row (horizontal).
__global__ void k_lns(float* __restrict__ out, int N, const int* __restrict__ kinds, float sigma, float period,
                      int nbrs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (i >= (long long)N * N) return;
  const int c = (int)(i / N), r = (int)(i - (long long)c * N);
  const float pos = (float)(kinds[b] == 0 ? c : r);
  const float centre = 0.5f * (float)(N - 1);
  const float den = __fmul_rn(2.f, __fmul_rn(sigma, sigma));
  float val = 0.f;
  for (int k = -nbrs; k <= nbrs; ++k) {
    const float dx = __fsub_rn(pos, __fadd_rn(centre, __fmul_rn((float)k, period)));
    val = __fadd_rn(val, expf(__fdiv_rn(-__fmul_rn(dx, dx), den)));
  }
  out[(long long)b * N * N + i] = __fsub_rn(val, 0.5f);
}

int next_pow2(int n) {
  int p = 1;
  while (p < n) p <<= 1;
  return p;
}

// Zero-padded taps hz[0 .. 2R+14]: hz[k] = h(R + 7 - k) for 7 <= k <= 2R+7,
// else 0, of the 1-D filters of the periodic covariance exp(-d^2/(2 ell^2))
// on Np points.  Its spectrum S(k) can dip below zero when the covariance
// is not negligible at d = Np/2; the 2-D filter sqrt(max(0, S(kx) S(ky)))
// is then Hp x Hp + Hn x Hn with Hp = sqrt(max(0, S)), Hn = sqrt(max(0, -S)):
// two separable filters (hzn empty when S >= 0).  Returns R, or -1 if the
// filter needs more than kMaxTaps taps.
int grf_taps(int Np, double ell, std::vector<float>& hzp, std::vector<float>& hzn) {
  const double two_pi = 6.283185307179586476925286766559;
  std::vector<double> ct(Np);
  for (int j = 0; j < Np; ++j) ct[j] = std::cos(two_pi * j / Np);
  // S(k) = sum over nearest-image d in (-Np/2, Np/2] of c(d) e^{-2 pi i k d / Np}
  const int D = std::min(Np / 2, (int)std::ceil(12.0 * ell));
  std::vector<double> c(D + 1);
  for (int d = 0; d <= D; ++d) c[d] = std::exp(-0.5 * (double)d * d / (ell * ell));
  std::vector<double> S(Np / 2 + 1), Hp(Np / 2 + 1), Hn(Np / 2 + 1);
  for (int k = 0; k <= Np / 2; ++k) {
    double s = c[0];
    for (int d = 1; d <= D; ++d) {
      const double term = c[d] * ct[(long long)k * d % Np];
      s += (2 * d == Np) ? term : 2.0 * term;  // d = Np/2 occurs once
    }
    S[k] = s;
  }
  // negative values at the level of the summation's rounding are zeros
  // (their products in the 2-D filter are below 1e-24 of its peak)
  const double floor_s = 1e-12 * S[0];
  bool neg = false;
  for (int k = 0; k <= Np / 2; ++k) {
    Hp[k] = std::sqrt(std::max(0.0, S[k]));
    Hn[k] = S[k] < -floor_s ? std::sqrt(-S[k]) : 0.0;
    neg = neg || S[k] < -floor_s;
  }
  // h(d) = (1/Np) sum_k H(k) e^{2 pi i k d / Np}, H even in k
  auto h_at = [&](const std::vector<double>& H, int d) {
    double s = H[0] + H[Np / 2] * ((d & 1) ? -1.0 : 1.0);
    for (int k = 1; k < Np / 2; ++k) s += 2.0 * H[k] * ct[(long long)k * d % Np];
    return s / Np;
  };
  int R = 0;
  std::vector<double> hp(1, h_at(Hp, 0)), hn(1, h_at(Hn, 0));
  if (neg) {
    // the covariance wraps around: keep the whole period
    if (Np / 2 > (kMaxTaps - 1) / 2) return -1;
    for (R = 1; R <= Np / 2; ++R) {
      hp.push_back(h_at(Hp, R));
      hn.push_back(h_at(Hn, R));
    }
    R = Np / 2;
  } else {
    const int Rmax = std::min(Np / 2, (kMaxTaps - 1) / 2);
    while (R < Rmax) {
      const double v = h_at(Hp, R + 1);
      if (std::fabs(v) < 1e-9 * hp[0] && std::exp(-(double)(R + 1) * (R + 1) / (ell * ell)) < 1e-9) break;
      hp.push_back(v);
      ++R;
    }
    if (2 * R < Np && std::exp(-(double)(R + 1) * (R + 1) / (ell * ell)) > 1e-7) return -1;
  }
  // A kernel spanning the whole period: the taps +-Np/2 hit the same input,
  // so each carries half of h(Np/2) and the convolution stays exact.
  if (2 * R == Np) {
    hp[R] *= 0.5;
    if (neg) hn[R] *= 0.5;
  }
  hzp.assign(2 * R + 15, 0.f);
  for (int k = 7; k <= 2 * R + 7; ++k) hzp[k] = (float)hp[std::abs(R + 7 - k)];
  hzn.clear();
  if (neg) {
    hzn.assign(2 * R + 15, 0.f);
    for (int k = 7; k <= 2 * R + 7; ++k) hzn[k] = (float)hn[std::abs(R + 7 - k)];
  }
  return R;
}

srk_status grf_run(const float* noise_in, unsigned long long seed, bool gen, int B, int N, double ell, int minmax,
                   cudaStream_t s, float* out) {
  if (!out) return fail(SRK_ERR_INVALID_ARG, "output is NULL");
  if (B < 1 || B > 65535 || N < 4 || N > 65536)
    return fail(SRK_ERR_INVALID_ARG, "need 1 <= B <= 65535, 4 <= N <= 65536 (B=%d N=%d)", B, N);
  if (!(ell > 0.0) || !std::isfinite(ell)) return fail(SRK_ERR_INVALID_ARG, "ell=%g must be positive", ell);
  const int Np = next_pow2(N);
  std::vector<float> hzp, hzn;
  const int R = grf_taps(Np, ell, hzp, hzn);
  if (R < 0)
    return fail(SRK_ERR_UNSUPPORTED, "ell=%g is too long for N=%d (at most %d filter taps, %d-point period)", ell, N,
                kMaxTaps, Np);
  const bool two = !hzn.empty();  // second separable filter (see grf_taps)
  const size_t smx = sizeof(float) * ((size_t)2 * R + 15 + (size_t)(64 + 2 * R) * 32);
  const int Hy = 256 + 2 * R;
  const size_t smy = sizeof(float) * ((size_t)2 * R + 15 + (size_t)8 * (Hy + Hy / 8 + 1));
  if (smx > 48 * 1024) SRK_CUDA(cudaFuncSetAttribute(k_grf_conv_x, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
  if (smy > 48 * 1024) SRK_CUDA(cudaFuncSetAttribute(k_grf_conv_y, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
  const size_t per = sizeof(float) * ((gen ? (size_t)Np * Np : 0) + (size_t)N * Np);
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)B, ((size_t)512 << 20) / per));
  float* hzd = nullptr;
  float* noise = nullptr;
  float* t = nullptr;
  unsigned* mm = nullptr;
  const size_t nt = hzp.size();
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&hzd), 2 * nt * sizeof(float), s));
  SRK_CUDA(cudaMemcpyAsync(hzd, hzp.data(), nt * sizeof(float), cudaMemcpyHostToDevice, s));
  if (two) SRK_CUDA(cudaMemcpyAsync(hzd + nt, hzn.data(), nt * sizeof(float), cudaMemcpyHostToDevice, s));
  if (gen) SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&noise), sizeof(float) * (size_t)chunk * Np * Np, s));
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&t), sizeof(float) * (size_t)chunk * N * Np, s));
  if (minmax) {
    SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&mm), sizeof(unsigned) * 2 * (size_t)B, s));
    SRK_CUDA(cudaMemsetAsync(mm, 0xFF, sizeof(unsigned) * B, s));
    SRK_CUDA(cudaMemsetAsync(mm + B, 0x00, sizeof(unsigned) * B, s));
  }
  for (int b0 = 0; b0 < B; b0 += chunk) {
    const int nb = std::min(chunk, B - b0);
    const float* w = noise_in ? noise_in + (size_t)b0 * Np * Np : noise;
    if (gen) {
      const long long groups = (long long)Np * Np / 4;
      k_grf_noise<<<dim3((unsigned)((groups + kSynThreads - 1) / kSynThreads), nb), kSynThreads, 0, s>>>(noise, Np,
                                                                                                    seed, b0);
    }
    for (int f = 0; f < (two ? 2 : 1); ++f) {
      const bool last = f == (two ? 1 : 0);
      k_grf_conv_x<<<dim3((Np + 31) / 32, (N + 63) / 64, nb), kSynThreads, smx, s>>>(w, t, Np, N, R, hzd + f * nt);
      k_grf_conv_y<<<dim3((N + 255) / 256, (N + 7) / 8, nb), kSynThreads, smy, s>>>(
          t, out + (size_t)b0 * N * N, Np, N, R, hzd + f * nt, (mm && last) ? mm + b0 : nullptr, B, f);
    }
    SRK_CUDA(cudaGetLastError());
  }
  if (minmax) {
    // the min/max of image b live at mm[b] and mm[B + b]
    k_minmax_scale<<<dim3((unsigned)(((long long)N * N + kSynThreads - 1) / kSynThreads), B), kSynThreads, 0, s>>>(
        out, N, mm, B);
    SRK_CUDA(cudaGetLastError());
    SRK_CUDA(cudaFreeAsync(mm, s));
  }
  SRK_CUDA(cudaFreeAsync(t, s));
  if (noise) SRK_CUDA(cudaFreeAsync(noise, s));
  SRK_CUDA(cudaFreeAsync(hzd, s));
  return SRK_OK;
}

}  // namespace
}  // namespace srk

using namespace srk;

extern "C" {

srk_status srk_grf(int B, int N, double ell, unsigned long long seed, int minmax, srk_stream_t stream,
                   float* d_out) {
  g_last_error.clear();
  return grf_run(nullptr, seed, true, B, N, ell, minmax, stream, d_out);
}

srk_status srk_grf_filter(const float* d_noise, int B, int N, double ell, int minmax, srk_stream_t stream,
                          float* d_out) {
  g_last_error.clear();
  if (!d_noise) return fail(SRK_ERR_INVALID_ARG, "noise is NULL");
  return grf_run(d_noise, 0, false, B, N, ell, minmax, stream, d_out);
}

srk_status srk_lns(int B, int N, const int* kinds, float sigma_px, float period_px, int num_nbrs,
                   srk_stream_t stream, float* d_out) {
  g_last_error.clear();
  if (!d_out || !kinds) return fail(SRK_ERR_INVALID_ARG, "NULL pointer");
  if (B < 1 || B > 65535 || N < 1 || !(sigma_px > 0.f) || num_nbrs < 0 || num_nbrs > 1000)
    return fail(SRK_ERR_INVALID_ARG, "need 1 <= B <= 65535, N >= 1, sigma > 0, 0 <= num_nbrs <= 1000");
  for (int b = 0; b < B; ++b)
    if (kinds[b] != 0 && kinds[b] != 1) return fail(SRK_ERR_INVALID_ARG, "kinds[%d]=%d (0 vertical, 1 horizontal)", b, kinds[b]);
  // period 0 = 4 FWHM (gen_lns_vertical, test_pattern.cu:87-88), in the reference's float arithmetic
  const float fwhm = 2.f * sqrtf(2.f * logf(2.f)) * sigma_px;
  const float period = period_px > 0.f ? period_px : 4.f * fwhm;
  int* dk = nullptr;
  SRK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dk), sizeof(int) * B, stream));
  SRK_CUDA(cudaMemcpyAsync(dk, kinds, sizeof(int) * B, cudaMemcpyHostToDevice, stream));
  k_lns<<<dim3((unsigned)(((long long)N * N + kSynThreads - 1) / kSynThreads), B), kSynThreads, 0, stream>>>(
      d_out, N, dk, sigma_px, period, num_nbrs);
  SRK_CUDA(cudaGetLastError());
  SRK_CUDA(cudaFreeAsync(dk, stream));
  return SRK_OK;
}

}  // extern "C"
