// dropin_training.cu — a C++ caller written the way the reference's
// training/main_cd_training.cu op_test() slot is used, switched to the
// B200 library by including srk_b200.hpp.  Exits 0 on PASS, 1 on FAIL,
// like the reference's test executables.
//
// It builds the Green's tensor on the host (float A&S K1 form of
// make_kernel), its spectra through srk::srkPrecomputeKernelFreq, runs
// srk::srkTrainingForward on B smooth images with E = I, and checks every
// output pixel against a double-precision direct "valid" convolution on
// the host (max|d|/max|ref| < 1e-3, the forward criterion of
// adjoint/main_adjoint.cu:359-360).
#include <cmath>
#include <cstdio>
#include <vector>

#include "srk_b200.hpp"

static float k1_as(float x) {  // Abramowitz & Stegun 9.8.7 / 9.8.8
  if (x <= 2.f) {
    const float t = x / 3.75f, y = t * t, q = x * x * 0.25f;
    const float i1 = x * (0.5f + y * (0.87890594f + y * (0.51498869f + y * (0.15084934f + y * (0.02658733f +
                     y * (0.00301532f + y * 0.00032411f))))));
    const float p = 1.f + q * (0.15443144f - q * (0.67278579f + q * (0.18156897f + q * (0.01919402f +
                    q * (0.00110404f + q * 0.00004686f)))));
    return std::log(x * 0.5f) * i1 + p / x;
  }
  const float y = 2.f / x;
  const float p = 1.25331414f + y * (0.23498619f + y * (-0.03655620f + y * (0.01504268f + y * (-0.00780353f +
                  y * (0.00325614f - y * 0.00068245f)))));
  return std::exp(-x) / std::sqrt(x) * p;
}

int main() {
  const int N = 256, KW = 61, B = 3, e = (KW - 1) / 2, W = N - 2 * e;
  const float sigma = e / 3.f, gamma = 1.f / sigma, Rw = 3.f * sigma, dx = 1.f;
  std::vector<float> Kx(KW * KW, 0.f), Ky(KW * KW, 0.f);
  for (int i = 0; i < KW; ++i)
    for (int j = 0; j < KW; ++j) {
      const float x = (float)(i - KW / 2), y = (float)(j - KW / 2), r = std::sqrt(x * x + y * y);
      if (r < 1e-6f || r > Rw) continue;
      const float t = r / Rw;
      const float w = 0.42f + 0.5f * std::cos(3.14159265f * t) + 0.08f * std::cos(2.f * 3.14159265f * t);
      const float base = gamma / (2.f * 3.14159265f) * k1_as(gamma * r) * w;
      Kx[i * KW + j] = base * x / r;
      Ky[i * KW + j] = base * y / r;
    }
  std::vector<float> E((size_t)B * N * N);
  for (int b = 0; b < B; ++b)
    for (int c = 0; c < N; ++c)
      for (int r = 0; r < N; ++r)
        E[(size_t)b * N * N + (size_t)c * N + r] =
            0.5f + 0.25f * std::sin(0.05f * c + 0.3f * b) * std::cos(0.07f * r - 0.2f * b) + 0.1f * std::sin(0.011f * c * r);

  cudaStream_t stream;
  cudaStreamCreate(&stream);
  float *d_E, *d_R;
  cufftComplex *d_Gx, *d_Gy;
  cudaMalloc(&d_E, sizeof(float) * E.size());
  cudaMalloc(&d_R, sizeof(float) * (size_t)B * W * W);
  cudaMalloc(&d_Gx, sizeof(cufftComplex) * N * (N / 2 + 1));
  cudaMalloc(&d_Gy, sizeof(cufftComplex) * N * (N / 2 + 1));
  cudaMemcpy(d_E, E.data(), sizeof(float) * E.size(), cudaMemcpyHostToDevice);
  if (srk::srkPrecomputeKernelFreq(Kx, KW, KW, N, d_Gx, stream) != SRK_OK ||
      srk::srkPrecomputeKernelFreq(Ky, KW, KW, N, d_Gy, stream) != SRK_OK) {
    printf("FAIL: spectrum precompute: %s\n", srk_last_error());
    return 1;
  }
  srk::Workspace ws;
  const srk_status st = srk::srkTrainingForward(d_E, d_E, d_Gx, d_Gy, N, W, e, dx, B, stream, d_R, ws);
  if (st != SRK_OK) {
    printf("FAIL: srkTrainingForward: %s (%s)\n", srk_status_string(st), srk_last_error());
    return 1;
  }
  std::vector<float> R((size_t)B * W * W);
  cudaMemcpy(R.data(), d_R, sizeof(float) * R.size(), cudaMemcpyDeviceToHost);
  double worst = 0.0;
  for (int b = 0; b < B; ++b) {
    const float* I = E.data() + (size_t)b * N * N;
    double maxd = 0.0, maxr = 0.0;
    for (int ox = 0; ox < W; ++ox)
      for (int oy = 0; oy < W; ++oy) {
        const int gx = ox + e, gy = oy + e;
        double ux = 0.0, uy = 0.0;
        for (int kx = -KW / 2; kx <= KW / 2; ++kx)
          for (int ky = -KW / 2; ky <= KW / 2; ++ky) {
            const double v = I[(size_t)(gx - kx) * N + (gy - ky)];
            ux += v * Kx[(kx + KW / 2) * KW + ky + KW / 2];
            uy += v * Ky[(kx + KW / 2) * KW + ky + KW / 2];
          }
        const double ix = 0.5 * ((double)I[(size_t)(gx + 1) * N + gy] - I[(size_t)(gx - 1) * N + gy]);
        const double iy = 0.5 * ((double)I[(size_t)gx * N + gy + 1] - I[(size_t)gx * N + gy - 1]);
        const double ref = dx * dx * (ux * ix + uy * iy);
        maxd = std::fmax(maxd, std::fabs(ref - R[(size_t)b * W * W + (size_t)ox * W + oy]));
        maxr = std::fmax(maxr, std::fabs(ref));
      }
    worst = std::fmax(worst, maxd / maxr);
  }
  printf("%s: srkTrainingForward drop-in, B=%d N=%d KW=%d, max rel err %.3e\n", worst < 1e-3 ? "PASS" : "FAIL", B,
         N, KW, worst);
  cudaFree(d_E);
  cudaFree(d_R);
  cudaFree(d_Gx);
  cudaFree(d_Gy);
  cudaStreamDestroy(stream);
  return worst < 1e-3 ? 0 : 1;
}
