// Checks dsax::scaley_u8 (FP32 with an exact fallback) against the FP64
// form for every uint8 input over random and adversarial channel baselines.
// Prints "<checked> <mismatches> <slow-path count>".
#include <cstdio>
#include <cstdlib>
#include <random>

#include "dsax_scaley.h"

int main() {
  std::mt19937_64 rng(12345);
  std::uniform_real_distribution<float> us0(-20.f, 300.f), uvar(1e-3f, 5e4f), umn(0.f, 200.f),
      usig(0.1f, 40.f);
  long checked = 0, bad = 0, slow = 0;
  auto run = [&](float s0, float var0, float sig, float mn) {
    const double k = (double)sig / (double)sqrtf(var0);
    const float k2f = (float)(2.0 * k);
    for (int x = 0; x < 256; ++x) {
      const float xf = (float)x;
      const float f = dsax::scaley_u8(xf, s0, k2f, k, mn);
      const float e = dsax::scaley_u8_exact(xf, s0, k, mn);
      const float z = dsax::fma_rn(xf - s0, k2f, 2.0f * mn);
      const float h = z - floorf(z);
      if (!(fabsf(h - 0.5f) > (fabsf(z) + fabsf((xf - s0) * k2f) + 1.0f) * 4.76837158203125e-7f)) ++slow;
      ++checked;
      if (f != e) {
        if (bad < 10) printf("mismatch x=%d s0=%.9g var0=%.9g sig=%.9g mn=%.9g fast=%g exact=%g\n", x, s0, var0, sig, mn, f, e);
        ++bad;
      }
    }
  };
  for (int i = 0; i < 200000; ++i) run(us0(rng), uvar(rng), usig(rng), umn(rng));
  // the reference's constants (SIG 6, MN 48) over baselines near 64
  for (int i = 0; i < 200000; ++i) run(40.f + 0.001f * (float)i, 1.f + 0.01f * (float)(i % 4000), 6.f, 48.f);
  // exact ties of 2 val: k a power of two, s0 a quarter
  for (int e = -6; e <= 6; ++e)
    for (int q = -400; q <= 400; ++q) {
      const float k = ldexpf(1.f, e);
      const float var0 = (6.f / k) * (6.f / k);   // sqrtf(var0) = 6 / k exactly
      run(0.25f * (float)q, var0, 6.f, 48.f);
      run(0.25f * (float)q + 0.125f, var0, 6.f, 48.f);
    }
  printf("%ld %ld %ld\n", checked, bad, slow);
  return bad ? 1 : 0;
}
