// dsax_scaley.h -- scaley for uint8 filterbanks (src/gpu_flagger.cu:382-394)
// in FP32 with an exact fallback.  Host-compilable so that the CPU tests can
// check the fast form against the FP64 formula exhaustively.
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define DSAX_HD __host__ __device__ __forceinline__
#else
#define DSAX_HD inline
#endif

namespace dsax {

// float -> uint32, round to nearest even, saturating (0 for negative and
// NaN): the device's __float2uint_rn.
DSAX_HD uint32_t f2u_rn(float z) {
#if defined(__CUDA_ARCH__)
  return __float2uint_rn(z);
#else
  if (!(z > 0.0f)) return 0u;
  if (z >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)std::nearbyint((double)z);
#endif
}

DSAX_HD float fma_rn(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

// The reference's arithmetic: val = (x - s0) * k + MN with the difference
// in float and the rest in double, k = SIG / sqrtf(var0); the uint8 result
// is (float2uint_rn(2 val) / 2) mod 256.
DSAX_HD float scaley_u8_exact(float x, float s0, double k, float mn) {
  const float val = (float)((double)(x - s0) * k + (double)mn);
  return (float)((f2u_rn(2.0f * val) >> 1) & 255u);
}

// The same in FP32: z = (x - s0) * 2k + 2 MN with one rounding (k2f =
// float(2k)) is within 2^-23 (|z| + |(x - s0) 2k|) of 2 val (the errors of
// k2f, of the FMA and of val's own float rounding), so float2uint_rn(z) =
// float2uint_rn(2 val) unless z lies within four times that of a half
// integer, where the result could change; there (and for NaN or infinite
// z) the exact form is taken.
DSAX_HD float scaley_u8(float x, float s0, float k2f, double k, float mn) {
  const float f = x - s0;
  const float z = fma_rn(f, k2f, 2.0f * mn);
  const float h = z - floorf(z);
  const float tol = (fabsf(z) + fabsf(f * k2f) + 1.0f) * 4.76837158203125e-7f;   // 2^-21
  if (fabsf(h - 0.5f) > tol) return (float)((f2u_rn(z) >> 1) & 255u);
  return scaley_u8_exact(x, s0, k, mn);
}

}  // namespace dsax
