// ref_host.cpp — TEST INFRASTRUCTURE ONLY.  C entry points around the
// reference's own host-side input generators, compiled from the reference's
// sources where they lie (oracle/build.py).  Used to make golden inputs.
//   GpGenerator        third_party/include/stTestCore/gp_generator.h:95-254
//   generate_pattern   third_party/src/patternUtil/test_pattern.cu:162-175
#include <stTestCore/gp_generator.h>
#include <patternUtil/test_pattern.h>
#include <cstring>

extern "C" int ref_gp_field(int N, double ell, unsigned long long seed, float* out) {
  st::util::GpGenerator g(st::util::Covariance2D::isotropic(ell), N, N, seed);
  const std::vector<float> v = g.generate();
  std::memcpy(out, v.data(), sizeof(float) * v.size());
  return (int)v.size();
}

// kind: 0 = LNS vertical, 1 = LNS horizontal.  period 0 = auto (4 FWHM).
extern "C" int ref_lns(int kind, int N, float sigma_px, float period_px, float* out) {
  const st::util::TestPatternConfig cfg = kind == 0 ? st::util::TestPatternConfig::lns_vertical(N, sigma_px, period_px)
                                                    : st::util::TestPatternConfig::lns_horizontal(N, sigma_px, period_px);
  const std::vector<float> v = st::util::generate_pattern(cfg);
  std::memcpy(out, v.data(), sizeof(float) * v.size());
  return (int)v.size();
}
