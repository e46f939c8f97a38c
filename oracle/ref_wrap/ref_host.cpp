// ref_host.cpp — TEST INFRASTRUCTURE ONLY.  C entry points around the
// reference's own host-side input generators, compiled from the reference's
// sources where they lie (oracle/build.py).  Used to make golden inputs.
//   GpGenerator        third_party/include/stTestCore/gp_generator.h:95-254
//   generate_pattern   third_party/src/patternUtil/test_pattern.cu:162-175
#include <stTestCore/gp_generator.h>
#include <patternUtil/test_pattern.h>
#include <cstring>
#include <random>

extern "C" int ref_gp_field(int N, double ell, unsigned long long seed, float* out) {
  st::util::GpGenerator g(st::util::Covariance2D::isotropic(ell), N, N, seed);
  const std::vector<float> v = g.generate();
  std::memcpy(out, v.data(), sizeof(float) * v.size());
  return (int)v.size();
}

// The white noise GpGenerator::generate draws for this seed (the same
// engine, distribution and order: one std::normal_distribution per call,
// row-major over the padded Np x Np grid), written column-major
// out[c*Np + r], so that filtering it reproduces ref_gp_field.  Returns Np.
extern "C" int ref_gp_noise(int N, unsigned long long seed, double* out) {
  int Np = 1;
  while (Np < N) Np <<= 1;
  std::mt19937_64 rng(static_cast<std::mt19937_64::result_type>(seed));
  std::normal_distribution<double> normal(0.0, 1.0);
  for (int r = 0; r < Np; ++r)
    for (int c = 0; c < Np; ++c) out[(size_t)c * Np + r] = normal(rng);
  return Np;
}

// kind: 0 = LNS vertical, 1 = LNS horizontal.  period 0 = auto (4 FWHM).
extern "C" int ref_lns(int kind, int N, float sigma_px, float period_px, float* out) {
  const st::util::TestPatternConfig cfg = kind == 0 ? st::util::TestPatternConfig::lns_vertical(N, sigma_px, period_px)
                                                    : st::util::TestPatternConfig::lns_horizontal(N, sigma_px, period_px);
  const std::vector<float> v = st::util::generate_pattern(cfg);
  std::memcpy(out, v.data(), sizeof(float) * v.size());
  return (int)v.size();
}
