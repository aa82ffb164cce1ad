/*
 * hsi_oracle.c - TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A CPU restatement of the reference's per-frame detection path, kept in
 * double precision from end to end.  Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load it, and only as the thing results are
 * checked against; the library in hsi-detectors-cuda_b200/ never calls it.
 *
 * Reference behaviour followed (GokulEdakkePuram/hsi-detectors-cuda):
 *   SAM angle / best match / per-target maps   src/sam_cpu.cpp:13-77
 *   threshold + NMS + raster-order list         src/sam_cpu.cpp:86-138
 *   raw moments (lower triangle, double)        src/detectors_cpu.cpp:77-93,
 *                                               src/linalg.cpp:18-29
 *   mean / covariance / correlation             src/linalg.cpp:45-79
 *   shifted-moment rebuild                      src/linalg.cpp:81-103
 *   Cholesky / solve / triangular inverse       src/linalg.cpp:105-162
 *   detector statistics                         src/detector.cpp:47-152
 *   RX / ACE-best / CEM-best                    src/detectors_cpu.cpp:95-187
 *   chi-squared RX threshold                    src/detectors_cpu.cpp:52-75,189-206
 *   snapshot-mosaic demosaic                    src/hot_loader.cpp:144-182
 *
 * One deliberate difference: the reference narrows the detector statistics to
 * float before scoring (src/detector.cpp:11-17,83-84,125-127,144-145).  Here
 * they stay double, so these maps are the FP64 truth the GPU error is stated
 * against.  The reference itself (built from its own sources into oracle/_ref)
 * is the second, bit-faithful oracle.
 *
 * Parity of this restatement is pinned against the reference build through the
 * fixtures in tests/golden/ (see tests/test_oracle_golden.py).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../hsi-detectors-cuda_b200/csrc/synth.h"

#define ORC_API __attribute__((visibility("default")))

typedef struct orc_detection {
  int32_t x;
  int32_t y;
  int32_t target;
  float score;
} orc_detection;

/* ------------------------------------------------------------------------ */
/* SAM                                                                       */
/* ------------------------------------------------------------------------ */

/* Angle for one pixel and one target, given the target's norm
 * (src/sam_cpu.cpp:13-18): a directionless pixel or target is pi/2. */
static double orc_angle(double dot, double pixel_sq, double target_norm) {
  if (pixel_sq <= 0.0 || target_norm <= 0.0) return (double)1.57079632679489661923f;
  double c = dot / (sqrt(pixel_sq) * target_norm);
  if (c < -1.0) c = -1.0;
  if (c > 1.0) c = 1.0;
  return acos(c);
}

/* Per-target angle maps, target-major out[t * pixels + p]
 * (src/sam_cpu.cpp:22-46).  `stride` >= pixels is the BSQ plane stride. */
ORC_API void orc_sam_all(const float* cube, int64_t pixels, int64_t stride, int bands,
                         const float* targets, const float* norms, int num_targets,
                         float* out) {
  for (int64_t p = 0; p < pixels; ++p) {
    double sq = 0.0;
    for (int b = 0; b < bands; ++b) {
      const double v = cube[(int64_t)b * stride + p];
      sq += v * v;
    }
    for (int t = 0; t < num_targets; ++t) {
      double dot = 0.0;
      for (int b = 0; b < bands; ++b)
        dot += (double)cube[(int64_t)b * stride + p] * (double)targets[(int64_t)t * bands + b];
      out[(int64_t)t * pixels + p] = (float)orc_angle(dot, sq, norms[t]);
    }
  }
}

/* Best match over targets: smallest angle, lowest index on ties
 * (src/sam_cpu.cpp:48-77). */
ORC_API void orc_sam_best(const float* cube, int64_t pixels, int64_t stride, int bands,
                          const float* targets, const float* norms, int num_targets,
                          float* out_score, int32_t* out_target) {
  for (int64_t p = 0; p < pixels; ++p) {
    double sq = 0.0;
    for (int b = 0; b < bands; ++b) {
      const double v = cube[(int64_t)b * stride + p];
      sq += v * v;
    }
    double best = INFINITY;
    int32_t best_t = -1;
    for (int t = 0; t < num_targets; ++t) {
      double dot = 0.0;
      for (int b = 0; b < bands; ++b)
        dot += (double)cube[(int64_t)b * stride + p] * (double)targets[(int64_t)t * bands + b];
      const double a = orc_angle(dot, sq, norms[t]);
      if (a < best) {
        best = a;
        best_t = t;
      }
    }
    out_score[p] = (float)best;
    if (out_target) out_target[p] = best_t;
  }
}

/* Target norms as the reference's SpectralLibrary::norms computes them:
 * double accumulation, narrowed to float (src/types.cpp:69-80). */
ORC_API void orc_target_norms(const float* targets, int num_targets, int bands, float* out) {
  for (int t = 0; t < num_targets; ++t) {
    double acc = 0.0;
    for (int b = 0; b < bands; ++b) {
      const double v = targets[(int64_t)t * bands + b];
      acc += v * v;
    }
    out[t] = (float)sqrt(acc);
  }
}

/* ------------------------------------------------------------------------ */
/* Detection list                                                            */
/* ------------------------------------------------------------------------ */

static int orc_better(float a, float b, int higher) { return higher ? a > b : a < b; }

/* Strictly-better or equal-with-lower-index neighbour suppresses the pixel
 * (src/sam_cpu.cpp:95-112). */
static int orc_local_best(const float* s, int x, int y, int w, int h, int r, float self,
                          int higher) {
  const int64_t self_idx = (int64_t)y * w + x;
  for (int dy = -r; dy <= r; ++dy) {
    const int ny = y + dy;
    if (ny < 0 || ny >= h) continue;
    for (int dx = -r; dx <= r; ++dx) {
      if (dx == 0 && dy == 0) continue;
      const int nx = x + dx;
      if (nx < 0 || nx >= w) continue;
      const int64_t n = (int64_t)ny * w + nx;
      if (orc_better(s[n], self, higher)) return 0;
      if (s[n] == self && n < self_idx) return 0;
    }
  }
  return 1;
}

/* Threshold (<= for lower-is-better, >= for higher-is-better) and NMS, in
 * raster order (src/sam_cpu.cpp:116-138).  Writes at most `capacity` entries
 * and returns how many were found. */
ORC_API int64_t orc_detect(const float* score, const int32_t* target, int height, int width,
                           float threshold, int nms_radius, int higher_is_better,
                           orc_detection* out, int64_t capacity) {
  int64_t found = 0;
  for (int y = 0; y < height; ++y) {
    for (int x = 0; x < width; ++x) {
      const int64_t p = (int64_t)y * width + x;
      const float s = score[p];
      const int over = higher_is_better ? (s >= threshold) : (s <= threshold);
      if (!over) continue;
      if (nms_radius > 0 &&
          !orc_local_best(score, x, y, width, height, nms_radius, s, higher_is_better))
        continue;
      if (found < capacity) {
        out[found].x = x;
        out[found].y = y;
        out[found].target = target ? target[p] : 0;
        out[found].score = s;
      }
      ++found;
    }
  }
  return found;
}

/* ------------------------------------------------------------------------ */
/* Scene moments and statistics                                              */
/* ------------------------------------------------------------------------ */

/* Raw first and second moments in double.  `outer` receives the full
 * symmetric B x B matrix (the reference accumulates the lower triangle,
 * src/linalg.cpp:18-29, and mirrors on read, :56-66). */
ORC_API void orc_moments(const float* cube, int64_t pixels, int64_t stride, int bands,
                         double* sum, double* outer) {
  double* x = (double*)malloc(sizeof(double) * (size_t)bands);
  memset(sum, 0, sizeof(double) * (size_t)bands);
  memset(outer, 0, sizeof(double) * (size_t)bands * (size_t)bands);
  for (int64_t p = 0; p < pixels; ++p) {
    for (int b = 0; b < bands; ++b) x[b] = cube[(int64_t)b * stride + p];
    for (int i = 0; i < bands; ++i) {
      sum[i] += x[i];
      double* row = outer + (int64_t)i * bands;
      for (int j = 0; j <= i; ++j) row[j] += x[i] * x[j];
    }
  }
  for (int i = 0; i < bands; ++i)
    for (int j = 0; j < i; ++j) outer[(int64_t)j * bands + i] = outer[(int64_t)i * bands + j];
  free(x);
}

/* M1 = S1 + N r, M2 = S2 + r S1^T + S1 r^T + N r r^T from sums about a
 * reference point r (src/linalg.cpp:81-103).  Full symmetric output. */
ORC_API void orc_moments_from_shifted(const double* s1, const double* s2_lower, double count,
                                      const double* ref, int bands, double* sum,
                                      double* outer) {
  for (int i = 0; i < bands; ++i) sum[i] = s1[i] + count * ref[i];
  for (int i = 0; i < bands; ++i) {
    for (int j = 0; j <= i; ++j) {
      const double v = s2_lower[(int64_t)i * bands + j] + ref[i] * s1[j] + s1[i] * ref[j] +
                       count * ref[i] * ref[j];
      outer[(int64_t)i * bands + j] = v;
      outer[(int64_t)j * bands + i] = v;
    }
  }
}

/* In-place Cholesky of a row-major SPD matrix; strict upper triangle zeroed.
 * Returns 0 on failure (not positive definite, or NaN) (src/linalg.cpp:105-122). */
ORC_API int orc_cholesky(double* a, int n) {
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j <= i; ++j) {
      double s = a[(int64_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= a[(int64_t)i * n + k] * a[(int64_t)j * n + k];
      if (i == j) {
        if (!(s > 0.0)) return 0;
        a[(int64_t)i * n + i] = sqrt(s);
      } else {
        a[(int64_t)i * n + j] = s / a[(int64_t)j * n + j];
      }
    }
    for (int j = i + 1; j < n; ++j) a[(int64_t)i * n + j] = 0.0;
  }
  return 1;
}

/* Solve L L^T x = b (src/linalg.cpp:124-137). */
ORC_API void orc_cholesky_solve(const double* l, int n, const double* b, double* x) {
  for (int i = 0; i < n; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= l[(int64_t)i * n + k] * x[k];
    x[i] = s / l[(int64_t)i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int k = i + 1; k < n; ++k) s -= l[(int64_t)k * n + i] * x[k];
    x[i] = s / l[(int64_t)i * n + i];
  }
}

/* Column-by-column forward substitution for L^-1, strict upper zero
 * (src/linalg.cpp:150-162). */
ORC_API void orc_triangular_inverse_lower(const double* l, int n, double* inv) {
  memset(inv, 0, sizeof(double) * (size_t)n * (size_t)n);
  for (int k = 0; k < n; ++k) {
    inv[(int64_t)k * n + k] = 1.0 / l[(int64_t)k * n + k];
    for (int i = k + 1; i < n; ++i) {
      double s = 0.0;
      for (int j = k; j < i; ++j) s -= l[(int64_t)i * n + j] * inv[(int64_t)j * n + k];
      inv[(int64_t)i * n + k] = s / l[(int64_t)i * n + i];
    }
  }
}

/* Status codes of orc_build_statistics. */
#define ORC_STATS_OK 0
#define ORC_STATS_EMPTY 1
#define ORC_STATS_COVARIANCE_NOT_PD 2
#define ORC_STATS_CORRELATION_NOT_PD 3

/* Detector statistics from raw moments, all in double (src/detector.cpp:47-152):
 *   mean = M1/N;  S = M2/N - mu mu^T + loading*I = L L^T;  W = L^-1;
 *   per target: u_t = W (d_t - mu), |u_t|^2;  w_t = R^-1 d_t / (d_t^T R^-1 d_t)
 *   with R = M2/N + loading*I, and w_t = 0 when that gain is not positive.
 * `outer` is the full symmetric M2 (only the lower triangle is read). */
ORC_API int orc_build_statistics(const double* sum, const double* outer, double count,
                                 int bands, const float* targets, int num_targets,
                                 double loading, double* mean, double* whitener,
                                 double* target_white, double* target_norm2,
                                 double* cem_weight) {
  if (!(count > 0.0)) return ORC_STATS_EMPTY;
  const int n = bands;
  const size_t nn = (size_t)n * (size_t)n;
  double* cov = (double*)malloc(sizeof(double) * nn);
  double* cor = (double*)malloc(sizeof(double) * nn);
  double* tmp = (double*)malloc(sizeof(double) * 3 * (size_t)n);
  double* centred = tmp;
  double* raw = tmp + n;
  double* solved = tmp + 2 * n;
  int status = ORC_STATS_OK;

  for (int i = 0; i < n; ++i) mean[i] = sum[i] / count;
  /* correlation first, then covariance by subtracting mu mu^T
   * (src/linalg.cpp:56-79) */
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j <= i; ++j) {
      const double r = outer[(int64_t)i * n + j] / count;
      cor[(int64_t)i * n + j] = r;
      cor[(int64_t)j * n + i] = r;
      const double c = r - mean[i] * mean[j];
      cov[(int64_t)i * n + j] = c;
      cov[(int64_t)j * n + i] = c;
    }
    cor[(int64_t)i * n + i] += loading;
    cov[(int64_t)i * n + i] += loading;
  }
  if (!orc_cholesky(cov, n)) {
    status = ORC_STATS_COVARIANCE_NOT_PD;
    goto done;
  }
  orc_triangular_inverse_lower(cov, n, whitener);
  if (num_targets > 0 && !orc_cholesky(cor, n)) {
    status = ORC_STATS_CORRELATION_NOT_PD;
    goto done;
  }
  for (int t = 0; t < num_targets; ++t) {
    const float* d = targets + (int64_t)t * n;
    for (int i = 0; i < n; ++i) centred[i] = (double)d[i] - mean[i];
    double norm2 = 0.0;
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      const double* row = whitener + (int64_t)i * n;
      for (int j = 0; j <= i; ++j) s += row[j] * centred[j];
      target_white[(int64_t)t * n + i] = s;
      norm2 += s * s;
    }
    target_norm2[t] = norm2;
    for (int i = 0; i < n; ++i) raw[i] = d[i];
    orc_cholesky_solve(cor, n, raw, solved);
    double gain = 0.0;
    for (int i = 0; i < n; ++i) gain += raw[i] * solved[i];
    for (int i = 0; i < n; ++i) cem_weight[(int64_t)t * n + i] = gain > 0.0 ? solved[i] / gain : 0.0;
  }
done:
  free(cov);
  free(cor);
  free(tmp);
  return status;
}

/* ------------------------------------------------------------------------ */
/* RX / ACE / CEM                                                            */
/* ------------------------------------------------------------------------ */

/* z = W y over the lower triangle; returns |z|^2 (src/detectors_cpu.cpp:27-36). */
static double orc_whiten(const double* w, int n, const double* y, double* z) {
  double nrm = 0.0;
  for (int i = 0; i < n; ++i) {
    const double* row = w + (int64_t)i * n;
    double s = 0.0;
    for (int j = 0; j <= i; ++j) s += row[j] * y[j];
    z[i] = s;
    nrm += s * s;
  }
  return nrm;
}

/* RX = |W (x - mu)|^2 (src/detectors_cpu.cpp:95-113). */
ORC_API void orc_rx(const float* cube, int64_t pixels, int64_t stride, int bands,
                    const double* mean, const double* whitener, float* out) {
  double* y = (double*)malloc(sizeof(double) * 2 * (size_t)bands);
  double* z = y + bands;
  for (int64_t p = 0; p < pixels; ++p) {
    for (int b = 0; b < bands; ++b) y[b] = (double)cube[(int64_t)b * stride + p] - mean[b];
    out[p] = (float)orc_whiten(whitener, bands, y, z);
  }
  free(y);
}

/* ACE per target (double), best over targets with the reference's rules
 * (src/detectors_cpu.cpp:115-156): skip a target when |u|^2 <= 0 or |z|^2 <= 0,
 * strict '>' so the lowest index wins ties, score clamp(best, 0, 1) and target
 * -1 when nothing was valid.  `out_all` (nullable) gets every target's ACE,
 * target-major, 0 where skipped; `out_rx` (nullable) gets |z|^2. */
ORC_API void orc_ace(const float* cube, int64_t pixels, int64_t stride, int bands,
                     const double* mean, const double* whitener, const double* target_white,
                     const double* target_norm2, int num_targets, float* out_score,
                     int32_t* out_target, float* out_rx, float* out_all) {
  double* y = (double*)malloc(sizeof(double) * 2 * (size_t)bands);
  double* z = y + bands;
  for (int64_t p = 0; p < pixels; ++p) {
    for (int b = 0; b < bands; ++b) y[b] = (double)cube[(int64_t)b * stride + p] - mean[b];
    const double zz = orc_whiten(whitener, bands, y, z);
    if (out_rx) out_rx[p] = (float)zz;
    double best = -1.0;
    int32_t best_t = -1;
    for (int t = 0; t < num_targets; ++t) {
      const double uu = target_norm2[t];
      double score = 0.0;
      if (uu > 0.0 && zz > 0.0) {
        const double* u = target_white + (int64_t)t * bands;
        double zu = 0.0;
        for (int b = 0; b < bands; ++b) zu += z[b] * u[b];
        score = (zu * zu) / (uu * zz);
        if (score > best) {
          best = score;
          best_t = t;
        }
      }
      if (out_all) out_all[(int64_t)t * pixels + p] = (float)score;
    }
    if (out_score) out_score[p] = (float)(best < 0.0 ? 0.0 : (best > 1.0 ? 1.0 : best));
    if (out_target) out_target[p] = best_t;
  }
  free(y);
}

/* CEM response w_t . x on the uncentred pixel; best = max with strict '>'
 * from -inf (src/detectors_cpu.cpp:158-187).  `out_all` (nullable) gets every
 * target's response, target-major. */
ORC_API void orc_cem(const float* cube, int64_t pixels, int64_t stride, int bands,
                     const double* cem_weight, int num_targets, float* out_score,
                     int32_t* out_target, float* out_all) {
  for (int64_t p = 0; p < pixels; ++p) {
    double best = -INFINITY;
    int32_t best_t = -1;
    for (int t = 0; t < num_targets; ++t) {
      const double* w = cem_weight + (int64_t)t * bands;
      double r = 0.0;
      for (int b = 0; b < bands; ++b) r += w[b] * (double)cube[(int64_t)b * stride + p];
      if (r > best) {
        best = r;
        best_t = t;
      }
      if (out_all) out_all[(int64_t)t * pixels + p] = (float)r;
    }
    if (out_score) out_score[p] = (float)best;
    if (out_target) out_target[p] = best_t;
  }
}

/* ------------------------------------------------------------------------ */
/* Chi-squared threshold for RX                                             */
/* ------------------------------------------------------------------------ */

/* Regularised lower incomplete gamma P(a, x): power series for x < a + 1,
 * otherwise 1 - Q from the continued fraction evaluated by the modified Lentz
 * method (the standard published pair of expansions; the reference uses the
 * same split, src/detectors_cpu.cpp:52-75). */
static double orc_gamma_p(double a, double x) {
  if (x <= 0.0) return 0.0;
  const double log_prefactor = -x + a * log(x) - lgamma(a);
  if (x < a + 1.0) {
    double term = 1.0 / a, total = term;
    for (int n = 1; n < 1000; ++n) {
      term *= x / (a + n);
      total += term;
      if (fabs(term) < fabs(total) * 1e-16) break;
    }
    return total * exp(log_prefactor);
  }
  const double tiny = 1e-300;
  double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
  for (int n = 1; n < 1000; ++n) {
    const double an = -(double)n * ((double)n - a);
    b += 2.0;
    d = an * d + b;
    if (fabs(d) < tiny) d = tiny;
    c = b + an / c;
    if (fabs(c) < tiny) c = tiny;
    d = 1.0 / d;
    const double delta = d * c;
    h *= delta;
    if (fabs(delta - 1.0) < 1e-16) break;
  }
  return 1.0 - exp(log_prefactor) * h;
}

/* Threshold t with P(chi2_B > t) = rate, by bisection (src/detectors_cpu.cpp:189-206).
 * Returns NaN for invalid arguments (the reference throws). */
ORC_API double orc_rx_threshold(int bands, double rate) {
  if (bands <= 0 || !(rate > 0.0) || !(rate < 1.0)) return NAN;
  const double a = 0.5 * bands, want = 1.0 - rate;
  double lo = 0.0, hi = 4.0 * bands > 16.0 ? 4.0 * bands : 16.0;
  while (orc_gamma_p(a, 0.5 * hi) < want && hi < 1e9) hi *= 2.0;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    if (orc_gamma_p(a, 0.5 * mid) < want) lo = mid; else hi = mid;
  }
  return 0.5 * (lo + hi);
}

/* ------------------------------------------------------------------------ */
/* Demosaic                                                                  */
/* ------------------------------------------------------------------------ */

/* Raw (x, y) carries band (y % p) * p + (x % p) of spatial pixel (x/p, y/p),
 * optionally permuted by `order` (src/hot_loader.cpp:144-182).  Output BSQ,
 * (raw_h/p) x (raw_w/p) x bands, plane stride `stride`.  Returns 0 on bad
 * arguments. */
ORC_API int orc_demosaic(const float* raw, int raw_w, int raw_h, int period, int bands,
                         const int32_t* order, float* out, int64_t stride) {
  if (period <= 0 || bands <= 0 || bands > period * period) return 0;
  const int w = raw_w / period, h = raw_h / period;
  if (w <= 0 || h <= 0) return 0;
  for (int b = 0; b < bands; ++b) {
    const int pos = order ? order[b] : b;
    const int oy = pos / period, ox = pos % period;
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x)
        out[(int64_t)b * stride + (int64_t)y * w + x] =
            raw[(int64_t)(y * period + oy) * raw_w + (int64_t)x * period + ox];
  }
  return 1;
}

/* ------------------------------------------------------------------------ */
/* Host-side scene generator (test inputs)                                   */
/* ------------------------------------------------------------------------ */

/* Library spectra of a scene: n_end endmembers, then the targets, then the
 * anomaly spectrum, each `bands` floats. */
ORC_API void orc_scene_spectra(uint64_t library_seed, int bands, int n_end, int n_targets,
                               float* endmembers, float* targets, float* anomaly) {
  for (int k = 0; k < n_end; ++k)
    hsi_spectrum(library_seed, HSI_SPECTRUM_ENDMEMBER(k), bands, endmembers + (int64_t)k * bands);
  for (int t = 0; t < n_targets; ++t)
    hsi_spectrum(library_seed, HSI_SPECTRUM_TARGET(t), bands, targets + (int64_t)t * bands);
  if (anomaly) hsi_spectrum(library_seed, HSI_SPECTRUM_ANOMALY, bands, anomaly);
}

/* Generate pixels [pixel0, pixel0 + pixels) of a frame, BSQ with plane stride
 * `stride`.  `truth` (nullable) receives the per-pixel label. */
ORC_API void orc_generate(const hsi_scene_spec* spec, int64_t pixel0, int64_t pixels,
                          int64_t stride, float* cube, uint8_t* truth) {
  const int B = spec->bands;
  float* spectra = (float*)malloc(sizeof(float) * (size_t)B * (size_t)(spec->n_end + spec->n_targets + 1));
  float* em = spectra;
  float* tg = em + (int64_t)spec->n_end * B;
  float* an = tg + (int64_t)spec->n_targets * B;
  orc_scene_spectra(spec->library_seed, B, spec->n_end, spec->n_targets, em, tg, an);
  float col[8];
  for (int64_t i = 0; i < pixels; ++i) {
    const uint64_t p = (uint64_t)(pixel0 + i);
    const hsi_pixel_draw d = hsi_draw_pixel(spec, p);
    for (int b = 0; b < B; ++b) {
      for (int k = 0; k < spec->n_end; ++k) col[k] = em[(int64_t)k * B + b];
      float implant = 0.0f;
      if (d.implant >= 0) implant = d.implant < spec->n_targets ? tg[(int64_t)d.implant * B + b] : an[b];
      cube[(int64_t)b * stride + i] = hsi_pixel_value(spec, &d, p, b, col, implant);
    }
    if (truth) truth[i] = (uint8_t)d.truth;
  }
  free(spectra);
}

/* ------------------------------------------------------------------------ */
/* Learned screen: per-pixel MLP B -> 64 -> 32 -> 1 (no reference           */
/* counterpart; the FP64 checker of the device training and inference).      */
/* ------------------------------------------------------------------------ */
/*
 * Parameters (FP32 master copy), with Bp = bands rounded up to 64:
 *   W1[64][Bp] | b1[64] | W2[32][64] | b2[32] | w3[32] | b3
 * Forward:  h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2), z = w3 . h2 + b3.
 * Loss: mean over samples of w_s (softplus(z) - y z), w_s = pos_weight for
 * y = 1, else 1 (binary cross-entropy on the logit, positives weighted).
 * With round_bf16 the weights W1, W2, w3 are rounded to bfloat16 where they
 * are used and h1 is rounded to bfloat16 before the second layer -- the
 * device's numerics -- and the backward pass treats those roundings as the
 * identity (straight-through), like the device.  Features: [n][bands].
 */
#define ORC_H1 64
#define ORC_H2 32

static int orc_bp(int bands) { return (bands + 63) / 64 * 64; }

ORC_API int64_t orc_mlp_param_count(int bands) {
  return (int64_t)ORC_H1 * orc_bp(bands) + ORC_H1 + ORC_H2 * ORC_H1 + ORC_H2 + ORC_H2 + 1;
}

/* round-to-nearest-even to bfloat16, returned as a float */
static double orc_bf16(double v) {
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
  memcpy(&f, &u, 4);
  return (double)f;
}

static double orc_softplus(double z) { return z > 0.0 ? z + log1p(exp(-z)) : log1p(exp(z)); }

/* logits[n]; returns nothing.  With grads (count doubles, zeroed here) and
 * labels, also the loss gradient; returns the loss (0 without labels). */
ORC_API double orc_mlp(const float* params, int bands, const float* features, const float* labels, int n,
                       double pos_weight, int round_bf16, double* logits, double* grads) {
  const int B = bands, Bp = orc_bp(bands);
  const float* W1 = params;
  const float* b1 = W1 + (int64_t)ORC_H1 * Bp;
  const float* W2 = b1 + ORC_H1;
  const float* b2 = W2 + ORC_H2 * ORC_H1;
  const float* w3 = b2 + ORC_H2;
  const float* b3 = w3 + ORC_H2;
  double *gW1 = 0, *gb1 = 0, *gW2 = 0, *gb2 = 0, *gw3 = 0, *gb3 = 0;
  if (grads) {
    memset(grads, 0, sizeof(double) * (size_t)orc_mlp_param_count(bands));
    gW1 = grads;
    gb1 = gW1 + (int64_t)ORC_H1 * Bp;
    gW2 = gb1 + ORC_H1;
    gb2 = gW2 + ORC_H2 * ORC_H1;
    gw3 = gb2 + ORC_H2;
    gb3 = gw3 + ORC_H2;
  }
#define RW(v) (round_bf16 ? orc_bf16(v) : (double)(v))
  double loss = 0.0;
  for (int s = 0; s < n; ++s) {
    const float* x = features + (int64_t)s * B;
    double z1[ORC_H1], h1[ORC_H1], z2[ORC_H2], h2[ORC_H2];
    for (int j = 0; j < ORC_H1; ++j) {
      double a = b1[j];
      for (int b = 0; b < B; ++b) a += RW(W1[(int64_t)j * Bp + b]) * (double)x[b];
      z1[j] = a;
      h1[j] = a > 0.0 ? a : 0.0;
      if (round_bf16) h1[j] = orc_bf16(h1[j]);
    }
    for (int k = 0; k < ORC_H2; ++k) {
      double a = b2[k];
      for (int j = 0; j < ORC_H1; ++j) a += RW(W2[k * ORC_H1 + j]) * h1[j];
      z2[k] = a;
      h2[k] = a > 0.0 ? a : 0.0;
    }
    double z = b3[0];
    for (int k = 0; k < ORC_H2; ++k) z += RW(w3[k]) * h2[k];
    if (logits) logits[s] = z;
    if (!labels) continue;
    const double y = labels[s], w = y > 0.5 ? pos_weight : 1.0;
    loss += w * (orc_softplus(z) - y * z);
    if (!grads) continue;
    const double d3 = w * (1.0 / (1.0 + exp(-z)) - y) / n;
    gb3[0] += d3;
    double d2[ORC_H2], d1[ORC_H1];
    for (int k = 0; k < ORC_H2; ++k) {
      gw3[k] += d3 * h2[k];
      d2[k] = z2[k] > 0.0 ? d3 * RW(w3[k]) : 0.0;
      gb2[k] += d2[k];
      for (int j = 0; j < ORC_H1; ++j) gW2[k * ORC_H1 + j] += d2[k] * h1[j];
    }
    for (int j = 0; j < ORC_H1; ++j) {
      double a = 0.0;
      for (int k = 0; k < ORC_H2; ++k) a += d2[k] * RW(W2[k * ORC_H1 + j]);
      d1[j] = z1[j] > 0.0 ? a : 0.0;
      gb1[j] += d1[j];
      for (int b = 0; b < B; ++b) gW1[(int64_t)j * Bp + b] += d1[j] * (double)x[b];
    }
  }
#undef RW
  return labels ? loss / n : 0.0;
}
