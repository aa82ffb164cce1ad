// ref_shim.cpp - TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// extern "C" wrappers around the reference's own CPU scorer, compiled together
// with the reference sources (unmodified, from where they lie) into
// oracle/_ref/libhsi_ref.so by oracle/Makefile.  Python tests, the golden
// fixture script and bench.py's reference arm load it with ctypes.
//
// Every wrapper converts plain pointers into the reference's types and calls
// exactly one reference entry point:
//   ref_sam_best / ref_sam_all      hsi::sam_best_cpu / hsi::sam_cpu   (src/sam_cpu.cpp:22-77)
//   ref_detect                      hsi::detect_cpu                    (src/sam_cpu.cpp:116-138)
//   ref_moments                     hsi::accumulate_moments_cpu         (src/detectors_cpu.cpp:77-93)
//   ref_build_statistics            hsi::build_statistics               (src/detector.cpp:47-152)
//   ref_rx / ref_ace_best / ref_cem_best   (src/detectors_cpu.cpp:95-187)
//   ref_rx_threshold                hsi::rx_threshold_for_false_alarm_rate (:189-206)
//   ref_cholesky / ref_triangular_inverse_lower / ref_cholesky_solve /
//   ref_moments_from_shifted        src/linalg.cpp:81-162
//   ref_demosaic                    hsi::demosaic                       (src/hot_loader.cpp:144-182)
//   ref_synthetic_frame             hsi::make_synthetic_source          (src/frame_source.cpp:149-293)
//   ref_read_envi                   hsi::read_envi                      (src/envi.cpp:195-258)
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "hsi/detector.hpp"
#include "hsi/detectors.hpp"
#include "hsi/envi.hpp"
#include "hsi/frame_source.hpp"
#include "hsi/hot_loader.hpp"
#include "hsi/linalg.hpp"
#include "hsi/sam.hpp"
#include "hsi/types.hpp"

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

hsi::CubeShape shape_of(int h, int w, int b) {
  hsi::CubeShape s;
  s.height = h;
  s.width = w;
  s.bands = b;
  return s;
}

hsi::SpectralLibrary library_of(const float* targets, int num_targets, int bands) {
  hsi::SpectralLibrary lib;
  for (int t = 0; t < num_targets; ++t) {
    hsi::Spectrum s;
    s.name = "t" + std::to_string(t);
    s.values.assign(targets + static_cast<std::size_t>(t) * bands,
                    targets + static_cast<std::size_t>(t + 1) * bands);
    lib.targets.push_back(std::move(s));
  }
  return lib;
}

hsi::DetectorStatistics stats_of(int bands, int num_targets, const float* mean,
                                 const float* whitener, const float* target_white,
                                 const float* target_norm2, const float* cem_weight) {
  hsi::DetectorStatistics s;
  s.bands = bands;
  s.num_targets = num_targets;
  const std::size_t b = static_cast<std::size_t>(bands);
  const std::size_t tb = static_cast<std::size_t>(num_targets) * b;
  s.mean.assign(mean, mean + b);
  s.whitener.assign(whitener, whitener + b * b);
  if (num_targets > 0) {
    s.target_white.assign(target_white, target_white + tb);
    s.target_norm2.assign(target_norm2, target_norm2 + num_targets);
    s.cem_weight.assign(cem_weight, cem_weight + tb);
  }
  s.valid = true;
  return s;
}

void copy_error(const std::string& message, char* buf, int len) {
  if (!buf || len <= 0) return;
  std::strncpy(buf, message.c_str(), static_cast<std::size_t>(len - 1));
  buf[len - 1] = '\0';
}

}  // namespace

REF_API void ref_sam_best(const float* cube, int h, int w, int b, const float* targets,
                          const float* norms, int num_targets, float* score, int32_t* target) {
  hsi::sam_best_cpu(cube, shape_of(h, w, b), targets, norms, num_targets, score, target);
}

REF_API void ref_sam_all(const float* cube, int h, int w, int b, const float* targets,
                         const float* norms, int num_targets, float* out) {
  hsi::sam_cpu(cube, shape_of(h, w, b), targets, norms, num_targets, out);
}

REF_API void ref_library_norms(const float* targets, int num_targets, int bands, float* out) {
  const std::vector<float> n = library_of(targets, num_targets, bands).norms();
  std::memcpy(out, n.data(), n.size() * sizeof(float));
}

// Returns the number of detections; writes min(count, capacity) entries of
// {x, y, target, score} (16 bytes each, the reference's Detection layout).
REF_API int64_t ref_detect(const float* score, const int32_t* target, int h, int w,
                           float threshold, int nms_radius, int higher_is_better,
                           void* out, int64_t capacity) {
  hsi::DetectionParams p;
  p.threshold = threshold;
  p.nms_radius = nms_radius;
  p.polarity = higher_is_better ? hsi::ScorePolarity::HigherIsBetter
                                : hsi::ScorePolarity::LowerIsBetter;
  const std::vector<hsi::Detection> found = hsi::detect_cpu(score, target, shape_of(h, w, 1), p);
  const int64_t n = static_cast<int64_t>(found.size());
  const int64_t keep = n < capacity ? n : capacity;
  if (keep > 0) std::memcpy(out, found.data(), static_cast<std::size_t>(keep) * sizeof(hsi::Detection));
  return n;
}

// sum[B] and outer[B*B] exactly as SpectralMoments holds them (lower triangle
// of outer accumulated, upper left at zero).
REF_API void ref_moments(const float* cube, int h, int w, int b, double* sum, double* outer,
                         double* count) {
  hsi::SpectralMoments m;
  hsi::accumulate_moments_cpu(cube, shape_of(h, w, b), &m);
  std::memcpy(sum, m.sum.data(), m.sum.size() * sizeof(double));
  std::memcpy(outer, m.sum_outer.data(), m.sum_outer.size() * sizeof(double));
  *count = m.count;
}

// Returns 1 on success; 0 with a message in `err` on failure.  Outputs are the
// reference's float-narrowed statistics.
REF_API int ref_build_statistics(const double* sum, const double* outer, double count, int bands,
                                 const float* targets, int num_targets, double loading,
                                 float* mean, float* whitener, float* target_white,
                                 float* target_norm2, float* cem_weight, char* err, int err_len) {
  hsi::SpectralMoments m;
  m.reset(bands);
  m.count = count;
  std::memcpy(m.sum.data(), sum, static_cast<std::size_t>(bands) * sizeof(double));
  std::memcpy(m.sum_outer.data(), outer,
              static_cast<std::size_t>(bands) * static_cast<std::size_t>(bands) * sizeof(double));
  hsi::DetectorStatistics s;
  std::string message;
  const bool ok = hsi::build_statistics(m, library_of(targets, num_targets, bands), loading, &s,
                                        &message);
  if (!ok) {
    copy_error(message, err, err_len);
    return 0;
  }
  std::memcpy(mean, s.mean.data(), s.mean.size() * sizeof(float));
  std::memcpy(whitener, s.whitener.data(), s.whitener.size() * sizeof(float));
  if (num_targets > 0) {
    std::memcpy(target_white, s.target_white.data(), s.target_white.size() * sizeof(float));
    std::memcpy(target_norm2, s.target_norm2.data(), s.target_norm2.size() * sizeof(float));
    std::memcpy(cem_weight, s.cem_weight.data(), s.cem_weight.size() * sizeof(float));
  }
  return 1;
}

REF_API int ref_rx(const float* cube, int h, int w, int b, const float* mean,
                   const float* whitener, float* out) {
  try {
    hsi::rx_cpu(cube, shape_of(h, w, b), stats_of(b, 0, mean, whitener, nullptr, nullptr, nullptr),
                out);
    return 1;
  } catch (const std::exception&) {
    return 0;
  }
}

REF_API int ref_ace_best(const float* cube, int h, int w, int b, int num_targets,
                         const float* mean, const float* whitener, const float* target_white,
                         const float* target_norm2, float* score, int32_t* target, float* rx) {
  try {
    const hsi::DetectorStatistics s =
        stats_of(b, num_targets, mean, whitener, target_white, target_norm2, target_white);
    hsi::ace_best_cpu(cube, shape_of(h, w, b), s, score, target, rx);
    return 1;
  } catch (const std::exception&) {
    return 0;
  }
}

REF_API int ref_cem_best(const float* cube, int h, int w, int b, int num_targets,
                         const float* mean, const float* whitener, const float* cem_weight,
                         float* score, int32_t* target) {
  try {
    std::vector<float> zeros(static_cast<std::size_t>(num_targets) * b, 0.0f);
    std::vector<float> zn(static_cast<std::size_t>(num_targets), 0.0f);
    hsi::DetectorStatistics s =
        stats_of(b, num_targets, mean, whitener, zeros.data(), zn.data(), cem_weight);
    hsi::cem_best_cpu(cube, shape_of(h, w, b), s, score, target);
    return 1;
  } catch (const std::exception&) {
    return 0;
  }
}

REF_API double ref_rx_threshold(int bands, double rate) {
  try {
    return hsi::rx_threshold_for_false_alarm_rate(bands, rate);
  } catch (const std::exception&) {
    return -1.0;
  }
}

REF_API int ref_cholesky(double* a, int n) { return hsi::cholesky(a, n) ? 1 : 0; }

REF_API void ref_cholesky_solve(const double* l, int n, const double* b, double* x) {
  hsi::cholesky_solve(l, n, b, x);
}

REF_API void ref_triangular_inverse_lower(const double* l, int n, double* inv) {
  hsi::triangular_inverse_lower(l, n, inv);
}

REF_API void ref_moments_from_shifted(const double* s1, const double* s2_lower, double count,
                                      const double* reference, int bands, double* sum,
                                      double* outer) {
  hsi::SpectralMoments m;
  hsi::moments_from_shifted(s1, s2_lower, count, reference, bands, &m);
  std::memcpy(sum, m.sum.data(), m.sum.size() * sizeof(double));
  std::memcpy(outer, m.sum_outer.data(), m.sum_outer.size() * sizeof(double));
}

// Returns 1 and fills `out` (BSQ, packed) on success; 0 on a rejected argument.
REF_API int ref_demosaic(const float* raw, int raw_w, int raw_h, int period, int bands,
                         const int32_t* order, int order_len, float* out) {
  try {
    hsi::PngImage img;
    img.width = raw_w;
    img.height = raw_h;
    img.samples.assign(raw, raw + static_cast<std::size_t>(raw_w) * raw_h);
    std::vector<int> ord;
    if (order && order_len > 0) ord.assign(order, order + order_len);
    const hsi::HsiFrame f = hsi::demosaic(img, period, bands, ord);
    std::memcpy(out, f.data.data(), f.data.size() * sizeof(float));
    return 1;
  } catch (const std::exception&) {
    return 0;
  }
}

// Frame `frame_index` of the reference's synthetic video source, BSQ packed,
// with its truth mask and planted library (num_targets * bands floats).
REF_API int ref_synthetic_frame(int h, int w, int b, int num_targets, int target_radius,
                                uint64_t seed, int frame_index, float* cube, uint8_t* truth,
                                float* library) {
  try {
    hsi::SyntheticOptions o;
    o.shape = shape_of(h, w, b);
    o.num_targets = num_targets;
    o.target_radius = target_radius;
    o.seed = seed;
    auto src = hsi::make_synthetic_source(o);
    for (int i = 0; i <= frame_index; ++i) {
      if (!src->read_into(cube, o.shape.pixels(), nullptr)) return 0;
    }
    std::memcpy(truth, src->truth_mask(), o.shape.pixels());
    const std::vector<float> flat = src->library()->flatten();
    std::memcpy(library, flat.data(), flat.size() * sizeof(float));
    return 1;
  } catch (const std::exception&) {
    return 0;
  }
}

// Best-of-everything CPU step of the reference for one frame, used as the
// timed CPU baseline: SAM per-target maps + best, scene moments,
// build_statistics, CEM best, and the detection list.  Returns detections found.
REF_API int64_t ref_frame_sam_cem(const float* cube, int h, int w, int b, const float* targets,
                                  int num_targets, double loading, float threshold,
                                  int nms_radius, float* sam_maps, float* sam_best,
                                  int32_t* sam_target, float* cem_best, int32_t* cem_target,
                                  void* detections, int64_t capacity) {
  const hsi::CubeShape shape = shape_of(h, w, b);
  const hsi::SpectralLibrary lib = library_of(targets, num_targets, b);
  const std::vector<float> flat = lib.flatten();
  const std::vector<float> norms = lib.norms();
  hsi::sam_cpu(cube, shape, flat.data(), norms.data(), num_targets, sam_maps);
  hsi::sam_best_cpu(cube, shape, flat.data(), norms.data(), num_targets, sam_best, sam_target);
  hsi::SpectralMoments m;
  hsi::accumulate_moments_cpu(cube, shape, &m);
  hsi::DetectorStatistics s;
  std::string err;
  if (!hsi::build_statistics(m, lib, loading, &s, &err)) return -1;
  hsi::cem_best_cpu(cube, shape, s, cem_best, cem_target);
  hsi::DetectionParams p;
  p.threshold = threshold;
  p.nms_radius = nms_radius;
  const std::vector<hsi::Detection> found = hsi::detect_cpu(sam_best, sam_target, shape, p);
  const int64_t n = static_cast<int64_t>(found.size());
  const int64_t keep = n < capacity ? n : capacity;
  if (keep > 0) std::memcpy(detections, found.data(), static_cast<std::size_t>(keep) * 16);
  return n;
}

// The reference's CPU step for the RX + ACE path on one frame: moments,
// build_statistics, ACE best with the shared RX map.
REF_API int ref_frame_rx_ace(const float* cube, int h, int w, int b, const float* targets,
                             int num_targets, double loading, float* ace, int32_t* ace_target,
                             float* rx) {
  const hsi::CubeShape shape = shape_of(h, w, b);
  const hsi::SpectralLibrary lib = library_of(targets, num_targets, b);
  hsi::SpectralMoments m;
  hsi::accumulate_moments_cpu(cube, shape, &m);
  hsi::DetectorStatistics s;
  std::string err;
  if (!hsi::build_statistics(m, lib, loading, &s, &err)) return 0;
  hsi::ace_best_cpu(cube, shape, s, ace, ace_target, rx);
  return 1;
}

// The reference's read_envi of `hdr` into interleave `to` (0 BSQ, 1 BIL,
// 2 BIP).  dims = {height, width, bands, wavelength count}.  Returns 0 with
// data (capacity floats) and wavelengths (wl_capacity floats) filled, 2 when
// a capacity is too small (dims filled), 1 on an exception, whose message
// goes to err (err_len bytes, NUL-terminated).
REF_API int ref_read_envi(const char* hdr, int to, int* dims, float* data, int64_t capacity, float* wavelengths,
                          int wl_capacity, char* err, int err_len) {
  try {
    const hsi::HsiFrame f = hsi::read_envi(hdr, static_cast<hsi::Interleave>(to));
    dims[0] = f.shape.height;
    dims[1] = f.shape.width;
    dims[2] = f.shape.bands;
    dims[3] = static_cast<int>(f.wavelengths_nm.size());
    if (static_cast<int64_t>(f.data.size()) > capacity || dims[3] > wl_capacity) return 2;
    std::memcpy(data, f.data.data(), f.data.size() * sizeof(float));
    if (dims[3]) std::memcpy(wavelengths, f.wavelengths_nm.data(), f.wavelengths_nm.size() * sizeof(float));
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) {
      std::strncpy(err, e.what(), static_cast<std::size_t>(err_len) - 1);
      err[err_len - 1] = '\0';
    }
    return 1;
  }
}
