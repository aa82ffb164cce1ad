// hsi/detector.hpp - detector kinds and the statistics RX, ACE and CEM use.
//
// Drop-in for the reference's include/hsi/detector.hpp:23-99.
// build_statistics keeps its host signature, but the factorisation (Cholesky
// of the loaded covariance and autocorrelation, triangular inverse, whitened
// targets, CEM weights) runs in FP64 on the GPU (hsi_build_statistics); the
// result is narrowed to float exactly as the reference's DetectorStatistics.
#pragma once

#include <string>
#include <vector>

#include "hsi/linalg.hpp"
#include "hsi/types.hpp"

namespace hsi {

enum class Detector {
  Sam,
  Rx,
  Ace,
  Cem,
};

struct DetectorTraits {
  const char* name;
  bool needs_targets;
  bool needs_statistics;
  ScorePolarity polarity;
  bool compute_bound;
};

// SAM lower-is-better; RX, ACE and CEM higher-is-better
// (reference src/detector.cpp:21-33).
DetectorTraits traits_of(Detector detector);
const char* to_string(Detector detector);
bool parse_detector(const std::string& name, Detector* out);

struct DetectorStatistics {
  int bands = 0;
  int num_targets = 0;
  std::vector<float> mean;          // bands
  std::vector<float> whitener;      // bands x bands, row-major, lower triangular: L^-1 of the covariance
  std::vector<float> target_white;  // num_targets x bands: L^-1 (d_t - mean)
  std::vector<float> target_norm2;  // num_targets: |target_white_t|^2
  std::vector<float> cem_weight;    // num_targets x bands: R^-1 d_t / (d_t^T R^-1 d_t), 0 if the gain <= 0
  bool valid = false;
};

// false (with *error naming the loading or the band count, and out->valid =
// false) when the moments are empty, the library's band count differs, or
// a loaded matrix fails to factor.  Synchronous; uses the current device.
bool build_statistics(const SpectralMoments& moments, const SpectralLibrary& library, double diagonal_loading,
                      DetectorStatistics* out, std::string* error);

}  // namespace hsi
