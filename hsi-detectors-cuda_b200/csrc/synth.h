/*
 * synth.h - the synthetic hyperspectral scene model, as pure functions.
 *
 * The reference measures on synthetic video (src/frame_source.cpp:149-293,
 * a moving-disc generator).  The workloads this library is benchmarked on use
 * a different, better-mixed model, stated here once and used by both the
 * device generator (generate.cu) and the host-side test generator:
 *
 *   endmember / target / anomaly spectrum = sum of 3 Gaussian bumps over the
 *       bands: centre U(0,B), width U(5,30)*B/113 bands, height U(0.1,0.9);
 *   background pixel = Dirichlet(1) mix of `n_end` endmembers
 *       (abundance_k = -ln U_k, normalised);
 *   implanted target t (probability target_frac each): (1-a)*mix + a*target,
 *       a ~ U(0.2, 0.8);
 *   anomaly (probability anomaly_frac, only on non-target pixels):
 *       (1-a)*mix + a*anomaly, a ~ U(0.5, 1.0);
 *   value = gain * that + N(0, noise_sigma^2), gain ~ U(0.3, 1.2), clipped >= 0.
 *
 * Every random number is a counter-based hash of (seed, pixel, draw index), so
 * a pixel's spectrum does not depend on how the work is split across threads
 * or devices.  Only the transcendental functions (expf, logf, sincosf) may
 * differ by an ulp between host and device; tests that compare a GPU result
 * with a CPU one therefore always read the device-generated cube back.
 *
 * Plain C so that both nvcc and gcc accept it.
 */
#ifndef HSI_B200_SYNTH_H
#define HSI_B200_SYNTH_H

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define HSI_HD __host__ __device__ __forceinline__
#else
#define HSI_HD static inline
#endif

/* Truth labels written beside a generated cube. */
#define HSI_TRUTH_BACKGROUND 0u
#define HSI_TRUTH_ANOMALY 255u /* targets are 1 + target index */

typedef struct hsi_scene_spec {
  int bands;           /* B */
  int n_end;           /* background endmembers, <= 8 */
  int n_targets;       /* implanted library size, <= 64 */
  float target_frac;   /* per-target implant probability per pixel */
  float anomaly_frac;  /* anomaly probability per pixel */
  float noise_sigma;   /* additive Gaussian noise */
  uint64_t library_seed; /* spectra (endmembers, targets, anomaly) */
  uint64_t frame_seed;   /* per-pixel draws */
} hsi_scene_spec;

/* splitmix64 finaliser: a bijective 64-bit mix. */
HSI_HD uint64_t hsi_mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

/* Uniform on the open interval (0, 1), 24 bits, for draw `k` of item `item`. */
HSI_HD float hsi_unit(uint64_t seed, uint64_t item, uint32_t k) {
  const uint64_t h = hsi_mix64(seed ^ hsi_mix64(item * 0x100000001b3ULL + (uint64_t)k));
  return ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);
}

/* Same draw in double precision (53 bits), used for the small host-side
 * spectra so that host and device agree on them exactly. */
HSI_HD double hsi_unit_f64(uint64_t seed, uint64_t item, uint32_t k) {
  const uint64_t h = hsi_mix64(seed ^ hsi_mix64(item * 0x100000001b3ULL + (uint64_t)k));
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

/* Spectrum ids inside one library seed. */
#define HSI_SPECTRUM_ENDMEMBER(k) ((uint64_t)(k))
#define HSI_SPECTRUM_TARGET(t) ((uint64_t)(1000 + (t)))
#define HSI_SPECTRUM_ANOMALY ((uint64_t)(900))

/* One smooth spectrum: the sum of three Gaussian bumps.  Computed in double on
 * the host; callers store it as float. */
HSI_HD void hsi_spectrum(uint64_t library_seed, uint64_t id, int bands, float* out) {
  const double scale = (double)bands / 113.0;
  double c[3], w[3], h[3];
  for (int f = 0; f < 3; ++f) {
    c[f] = hsi_unit_f64(library_seed, id, (uint32_t)(3 * f + 0)) * (double)bands;
    w[f] = (5.0 + 25.0 * hsi_unit_f64(library_seed, id, (uint32_t)(3 * f + 1))) * scale;
    h[f] = 0.1 + 0.8 * hsi_unit_f64(library_seed, id, (uint32_t)(3 * f + 2));
  }
  for (int b = 0; b < bands; ++b) {
    double v = 0.0;
    for (int f = 0; f < 3; ++f) {
      const double d = ((double)b - c[f]) / w[f];
      v += h[f] * exp(-0.5 * d * d);
    }
    out[b] = (float)v;
  }
}

/* Per-pixel draws that do not depend on the band. */
typedef struct hsi_pixel_draw {
  float abundance[8]; /* normalised, n_end used */
  float gain;
  float alpha;   /* weight of the implanted spectrum, 0 for plain background */
  int implant;   /* -1 none, 0..T-1 target, T = anomaly */
  unsigned truth;
} hsi_pixel_draw;

HSI_HD hsi_pixel_draw hsi_draw_pixel(const hsi_scene_spec* s, uint64_t pixel) {
  hsi_pixel_draw d;
  float total = 0.0f;
  for (int k = 0; k < 8; ++k) {
    float a = 0.0f;
    if (k < s->n_end) a = -logf(hsi_unit(s->frame_seed, pixel, (uint32_t)k));
    d.abundance[k] = a;
    total += a;
  }
  const float inv = 1.0f / total;
  for (int k = 0; k < 8; ++k) d.abundance[k] *= inv;
  d.gain = 0.3f + 0.9f * hsi_unit(s->frame_seed, pixel, 8u);
  d.alpha = 0.0f;
  d.implant = -1;
  d.truth = HSI_TRUTH_BACKGROUND;
  const float ut = hsi_unit(s->frame_seed, pixel, 9u);
  if (s->n_targets > 0 && ut < s->target_frac * (float)s->n_targets) {
    int t = (int)(ut / s->target_frac);
    if (t >= s->n_targets) t = s->n_targets - 1;
    d.implant = t;
    d.alpha = 0.2f + 0.6f * hsi_unit(s->frame_seed, pixel, 10u);
    d.truth = 1u + (unsigned)t;
  } else if (hsi_unit(s->frame_seed, pixel, 11u) < s->anomaly_frac) {
    d.implant = s->n_targets;
    d.alpha = 0.5f + 0.5f * hsi_unit(s->frame_seed, pixel, 12u);
    d.truth = HSI_TRUTH_ANOMALY;
  }
  return d;
}

/* Standard normal for band `band` of `pixel` (Box-Muller on a pair of draws
 * shared by bands 2i and 2i+1). */
HSI_HD float hsi_noise(const hsi_scene_spec* s, uint64_t pixel, int band) {
  const uint32_t pair = 16u + 2u * (uint32_t)(band >> 1);
  const float u1 = hsi_unit(s->frame_seed, pixel, pair);
  const float u2 = hsi_unit(s->frame_seed, pixel, pair + 1u);
  const float r = sqrtf(-2.0f * logf(u1));
  const float theta = 6.283185307179586f * u2;
  return (band & 1) ? r * sinf(theta) : r * cosf(theta);
}

/* Value of one band of one pixel, given the band's column of spectra:
 * endmember[k] for k < n_end, then the implanted spectrum value (ignored when
 * draw->implant < 0). */
HSI_HD float hsi_pixel_value(const hsi_scene_spec* s, const hsi_pixel_draw* d,
                             uint64_t pixel, int band, const float* endmember_col,
                             float implant_value) {
  float mix = 0.0f;
  for (int k = 0; k < s->n_end; ++k) mix = fmaf(d->abundance[k], endmember_col[k], mix);
  if (d->implant >= 0) mix = (1.0f - d->alpha) * mix + d->alpha * implant_value;
  float v = d->gain * mix + s->noise_sigma * hsi_noise(s, pixel, band);
  return v > 0.0f ? v : 0.0f;
}

#endif /* HSI_B200_SYNTH_H */
