// hsi/linalg.hpp - the moments container of the detector statistics.
//
// Drop-in for SpectralMoments of the reference's include/hsi/linalg.hpp:22-51
// (raw FP64 first and second moments and the count).  The accumulation over a
// frame's pixels runs on the GPU (hsi::accumulate_moments in
// hsi/detectors.hpp); the factorisations the reference does here on the host
// (Cholesky, triangular inverse, solves) run on the GPU inside
// hsi::build_statistics.
#pragma once

#include <cstddef>
#include <vector>

namespace hsi {

struct SpectralMoments {
  int bands = 0;
  double count = 0.0;
  std::vector<double> sum;        // M1, `bands` entries
  std::vector<double> sum_outer;  // M2, row-major bands x bands, symmetric

  void reset(int bands);
  // Add one spectrum (`bands` floats): M1 += x, M2 += x x^T, count += 1.
  void add(const float* spectrum);
  void merge(const SpectralMoments& other);
  bool empty() const { return count <= 0.0; }
  std::vector<double> mean() const;
  // M2/N - mean mean^T + loading * I
  std::vector<double> covariance(double diagonal_loading = 0.0) const;
  // M2/N + loading * I
  std::vector<double> correlation(double diagonal_loading = 0.0) const;
};

// Raw moments from sums about a reference spectrum (S1 = sum(x - r), S2 the
// lower triangle of sum (x - r)(x - r)^T, row-major), as
// src/linalg.cpp:81-103 of the reference.
void moments_from_shifted(const double* s1, const double* s2_lower, double count, const double* reference,
                          int bands, SpectralMoments* out);

}  // namespace hsi
