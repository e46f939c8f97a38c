// spectra.cuh — FP64 device kernels for the Green's tensor and its spectra.
//
// Conventions (matching srkPrecomputeKernelFreq, srk_forward.cuh:154-203):
//   * a spatial kernel K of width KW = 2c+1 is column-major K[i*KW + j],
//     column offset dx = i - c, row offset dy = j - c;
//   * its spectrum at size M is the unnormalised DFT of K wrapped so that the
//     centre sits at index 0:  G(ky,kx) = sum K(dx,dy) exp(-2 pi i (kx dx + ky dy)/M);
//   * reference layout ("R2C of the column-major buffer"): half spectrum
//     ref[kx*(M/2+1) + ky], ky in [0, M/2];
//   * engine layout: full spectrum full[ky*M + kx] (Hermitian extension).
// Twiddles exp(-2 pi i m/M) come from a double table indexed by (a*b) mod M,
// so no angle is ever reduced in floating point.
#pragma once
#include <cuda_runtime.h>
#include "fft_warp.cuh"

namespace srk {

// exp(-2 pi i m / M) from a table tab[m] = (cos, sin)(2 pi m / M).
__device__ __forceinline__ double2 tw64(const double2* __restrict__ tab, long long m, int M, double sign) {
  long long r = m % M;
  if (r < 0) r += M;
  const double2 t = tab[r];
  return make_double2(t.x, sign * t.y);
}

// Modified Bessel function K1(x), x > 0, by the trapezoidal rule applied to
// the integral representation K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt
// (DLMF 10.32.9, nu = 1).  The integrand is even and analytic in the strip
// |Im t| < pi/2, so the rule with step h converges like exp(-pi^2/h); h = 1/16
// is far below double rounding.  Terms are summed until they are negligible.
__device__ inline double bessel_k1(double x) {
  const double h = 1.0 / 16.0;
  double sum = 0.5 * exp(-x);  // t = 0 term, cosh(0) = 1
  for (int n = 1; n < 4096; ++n) {
    const double t = n * h;
    const double ch = cosh(t);
    const double term = exp(-x * ch) * ch;
    sum += term;
    if (term < 1e-19 * sum) break;
  }
  return h * sum;
}

// Green's tensor Gx = (gamma/2 pi)(x/r) K1(gamma r) w(r), Gy likewise with y,
// w = radial Blackman 0.42 + 0.5 cos(pi r/Rw) + 0.08 cos(2 pi r/Rw), zero for
// r > Rw and for r < 1e-6 dx (make_kernel, training/main_cd_training.cu:40-77;
// make_srsrk_kernel_2d, tan_tanadj/main_tan_tanadj.cu:93-116), in FP64.
__global__ void k_green_tensor(int KW, double gamma, double Rw, double dx, float* __restrict__ Kx,
                               float* __restrict__ Ky) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= KW * KW) return;
  const int i = idx / KW, j = idx - (idx / KW) * KW;
  const int c = KW / 2;
  const double x = (i - c) * dx, y = (j - c) * dx;
  const double r = sqrt(x * x + y * y);
  double gx = 0.0, gy = 0.0;
  if (!(r < 1e-6 * dx || r > Rw)) {
    const double t = r / Rw;
    const double w = 0.42 + 0.5 * cospi(t) + 0.08 * cospi(2.0 * t);
    const double base = gamma / (2.0 * 3.14159265358979323846) * bessel_k1(gamma * r) * w;
    gx = base * (x / r);
    gy = base * (y / r);
  }
  Kx[idx] = (float)gx;
  Ky[idx] = (float)gy;
}

// Pass 1 of the kernel DFT: P[j][kx] = sum_i K[i*KW+j] exp(-2 pi i kx (i-c)/M).
// The kernel is given in double (Kd) — the float path converts first.
__global__ void k_dft_cols(const double* __restrict__ Kd, int KW, int M, const double2* __restrict__ tab,
                           double2* __restrict__ P) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (kx >= M) return;
  const int c = KW / 2;
  double re = 0.0, im = 0.0;
  for (int i = 0; i < KW; ++i) {
    const double k = Kd[(long long)i * KW + j];
    if (k == 0.0) continue;
    const double2 w = tw64(tab, (long long)kx * (i - c), M, -1.0);
    re += k * w.x;
    im += k * w.y;
  }
  P[(long long)j * M + kx] = make_double2(re, im);
}

// Pass 2: G(ky,kx) = sum_j P[j][kx] exp(-2 pi i ky (j-c)/M); writes the
// engine layout scaled by `scale` (if full != null) and the reference layout
// unscaled (if ref != null).
__global__ void k_dft_rows(const double2* __restrict__ P, int KW, int M, const double2* __restrict__ tab,
                           double scale, float2* __restrict__ full, float2* __restrict__ ref) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ky = blockIdx.y;
  if (kx >= M) return;
  const int c = KW / 2;
  double re = 0.0, im = 0.0;
  for (int j = 0; j < KW; ++j) {
    const double2 p = P[(long long)j * M + kx];
    const double2 w = tw64(tab, (long long)ky * (j - c), M, -1.0);
    re += p.x * w.x - p.y * w.y;
    im += p.x * w.y + p.y * w.x;
  }
  if (full) full[(long long)ky * M + kx] = make_float2((float)(re * scale), (float)(im * scale));
  if (ref && ky <= M / 2) ref[(long long)kx * (M / 2 + 1) + ky] = make_float2((float)re, (float)im);
}

// Re-layout a reference half spectrum of size M into the engine layout with
// Hermitian extension: G(ky,kx) = conj(G(M-ky, M-kx)) for ky > M/2.
__global__ void k_relayout(const float2* __restrict__ ref, int M, float scale, float2* __restrict__ full) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ky = blockIdx.y;
  if (kx >= M) return;
  const int H = M / 2 + 1;
  float2 v;
  if (ky <= M / 2) {
    v = ref[(long long)kx * H + ky];
  } else {
    const float2 s = ref[(long long)((M - kx) % M) * H + (M - ky)];
    v = make_float2(s.x, -s.y);
  }
  full[(long long)ky * M + kx] = make_float2(v.x * scale, v.y * scale);
}

// Spatial recovery from a reference half spectrum of size Mr, restricted to
// offsets |dx|,|dy| <= c (the kernel support).  Pass A:
//   Tm[ky][dxi] = sum_kx ref(ky,kx) exp(+2 pi i kx dx / Mr),  dx = dxi - c.
__global__ void k_recover_a(const float2* __restrict__ ref, int Mr, int c, const double2* __restrict__ tab,
                            double2* __restrict__ Tm) {
  const int dxi = blockIdx.x * blockDim.x + threadIdx.x;
  const int ky = blockIdx.y;
  const int KW = 2 * c + 1;
  if (dxi >= KW) return;
  const int H = Mr / 2 + 1;
  const int dx = dxi - c;
  double re = 0.0, im = 0.0;
  for (int kx = 0; kx < Mr; ++kx) {
    const float2 g = ref[(long long)kx * H + ky];
    const double2 w = tw64(tab, (long long)kx * dx, Mr, +1.0);
    re += (double)g.x * w.x - (double)g.y * w.y;
    im += (double)g.x * w.y + (double)g.y * w.x;
  }
  Tm[(long long)ky * KW + dxi] = make_double2(re, im);
}

// Pass B: K(dx,dy) = Mr^-2 [T(0) + 2 sum_{ky=1}^{Mr/2-1} Re(T(ky) e^{+2 pi i ky dy/Mr}) + Re(T(Mr/2) (-1)^dy)]
// using T(-ky, dx) = conj(T(ky, dx)) for a real kernel.  Output column-major Kd[dxi*KW + dyi].
__global__ void k_recover_b(const double2* __restrict__ Tm, int Mr, int c, const double2* __restrict__ tab,
                            double* __restrict__ Kd) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int KW = 2 * c + 1;
  if (idx >= KW * KW) return;
  const int dxi = idx / KW, dyi = idx - (idx / KW) * KW;
  const int dy = dyi - c;
  double s = Tm[dxi].x;
  for (int ky = 1; ky < Mr / 2; ++ky) {
    const double2 t = Tm[(long long)ky * KW + dxi];
    const double2 w = tw64(tab, (long long)ky * dy, Mr, +1.0);
    s += 2.0 * (t.x * w.x - t.y * w.y);
  }
  const double2 tn = Tm[(long long)(Mr / 2) * KW + dxi];
  s += ((dy & 1) ? -1.0 : 1.0) * tn.x;
  Kd[idx] = s / ((double)Mr * (double)Mr);
}


// Double-precision twiddle table tab[m] = (cos, sin)(2 pi m / M), built on
// the device (sincospi takes the angle as a multiple of pi, so no angle is
// reduced in floating point): callers need no host table and no host sync.
__global__ void k_twiddles64(double2* __restrict__ tab, int M) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  double s, c;
  sincospi(2.0 * (double)m / (double)M, &s, &c);
  tab[m] = make_double2(c, s);
}

// The FFT engine's float twiddle table (per-pass blocks of tw_entry):
// exp(-2 pi i num/den) in double, rounded once to float; entries past
// tw_entries(M) are zero.  Plans and the no-allocation forward both build
// their tables with this kernel, so the two paths use identical twiddles.
__global__ void k_fft_twiddles(float2* __restrict__ tw, int M) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  float2 v = make_float2(0.f, 0.f);
  if (m < tw_entries(M)) {
    int num = 0, den = 1;
    tw_entry(M, m, num, den);
    double s, c;
    sincospi(2.0 * (double)num / (double)den, &s, &c);
    v = make_float2((float)c, (float)-s);
  }
  tw[m] = v;
}

// A KW x KW float kernel centred on a KWp x KWp support (KWp >= KW, both
// odd), in double, zero elsewhere; column-major both.
__global__ void k_pad_centre(const float* __restrict__ K, int KW, int KWp, double* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= KWp * KWp) return;
  const int i = idx / KWp - (KWp - KW) / 2, j = idx - (idx / KWp) * KWp - (KWp - KW) / 2;
  out[idx] = (i >= 0 && i < KW && j >= 0 && j < KW) ? (double)K[i * KW + j] : 0.0;
}

__global__ void k_float_to_double(const float* __restrict__ a, double* __restrict__ b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

}  // namespace srk
