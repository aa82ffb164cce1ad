// sam_math.cuh - the spectral-angle arithmetic shared by the SAM scorers.
//
// Every SAM kernel turns a cosine into an angle with these functions, so the
// BSQ and BIP scorers give bit-identical angles for the same dot products.
#pragma once

#include "common.cuh"

namespace hsi_b200 {

// Angle of a cosine clamped to [-1, 1] (a NaN clamps to -1, as with fminf/fmaxf).
// arccos by Abramowitz & Stegun 4.4.46 (Hastings' approximation):
//   acos(x) = sqrt(1 - x) (a0 + a1 x + ... + a7 x^7) + e(x),  |e| <= 2e-8 on [0, 1],
// and acos(-x) = pi - acos(x).  In FP32 the result is within a few 1e-7 rad of
// the exact angle, far inside the scorer's tolerances, at about half the
// instructions of the library arccos; sqrt(y) is y rsqrt(y) (y = 0 gives 0).
__device__ __forceinline__ float angle_of_cos(float c) {
  c = fminf(fmaxf(c, -1.0f), 1.0f);
  const float x = fabsf(c);
  float p = -0.0012624911f;
  p = fmaf(p, x, 0.0066700901f);
  p = fmaf(p, x, -0.0170881256f);
  p = fmaf(p, x, 0.0308918810f);
  p = fmaf(p, x, -0.0501743046f);
  p = fmaf(p, x, 0.0889789874f);
  p = fmaf(p, x, -0.2145988016f);
  p = fmaf(p, x, 1.5707963050f);
  const float y = 1.0f - x;
  const float r = y > 0.0f ? y * rsqrtf(y) * p : 0.0f;
  return c < 0.0f ? 3.14159265358979f - r : r;
}

// The same arccos for two cosines at once: the polynomial on the packed FMA
// pipe (each lane rounded as its own fmaf, so both lanes equal angle_of_cos).
__device__ __forceinline__ float2 angle_of_cos2(float2 c) {
  c.x = fminf(fmaxf(c.x, -1.0f), 1.0f);
  c.y = fminf(fmaxf(c.y, -1.0f), 1.0f);
  const float2 x = make_float2(fabsf(c.x), fabsf(c.y));
  float2 p = make_float2(-0.0012624911f, -0.0012624911f);
  p = ffma2(p, x, make_float2(0.0066700901f, 0.0066700901f));
  p = ffma2(p, x, make_float2(-0.0170881256f, -0.0170881256f));
  p = ffma2(p, x, make_float2(0.0308918810f, 0.0308918810f));
  p = ffma2(p, x, make_float2(-0.0501743046f, -0.0501743046f));
  p = ffma2(p, x, make_float2(0.0889789874f, 0.0889789874f));
  p = ffma2(p, x, make_float2(-0.2145988016f, -0.2145988016f));
  p = ffma2(p, x, make_float2(1.5707963050f, 1.5707963050f));
  const float yx = 1.0f - x.x, yy = 1.0f - x.y;
  const float rx = yx > 0.0f ? yx * rsqrtf(yx) * p.x : 0.0f;
  const float ry = yy > 0.0f ? yy * rsqrtf(yy) * p.y : 0.0f;
  return make_float2(c.x < 0.0f ? 3.14159265358979f - rx : rx, c.y < 0.0f ? 3.14159265358979f - ry : ry);
}

}  // namespace hsi_b200
