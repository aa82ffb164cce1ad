// The statistics and RX / ACE / CEM properties of the reference's detector
// tests, through the drop-in API on the device: hsi::build_statistics (FP64
// factorisation on the GPU), hsi::DeviceStatistics, hsi::launch_rx_ace,
// hsi::launch_cem and the stats_cuda accumulators.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "check.hpp"
#include "hsi/detector.hpp"
#include "hsi/detectors.hpp"
#include "hsi/frame_source.hpp"
#include "hsi/sam_cuda.hpp"
#include "hsi/stats_cuda.hpp"

using namespace hsi;
using tcheck::Dev;

namespace {

struct Scene {
  CubeShape shape;
  std::vector<float> host;  // at bsq_plane_stride
  std::vector<std::uint8_t> truth;
  SpectralLibrary library;
};

Scene make_scene(int h, int w, int b, int targets, float anomaly, std::uint64_t seed) {
  SyntheticOptions o;
  o.shape.height = h;
  o.shape.width = w;
  o.shape.bands = b;
  o.num_targets = targets;
  o.target_fraction = 0.003f;
  o.anomaly_fraction = anomaly;
  o.seed = seed;
  std::unique_ptr<FrameSource> src = make_synthetic_source(o);
  Scene s;
  s.shape = o.shape;
  s.host.resize(bsq_device_elements(o.shape));
  FrameMeta meta;
  CHECK(src->read_into(s.host.data(), bsq_plane_stride(o.shape), &meta));
  s.truth.assign(src->truth_mask(), src->truth_mask() + o.shape.pixels());
  s.library = *src->library();
  return s;
}

SpectralMoments host_moments(const Scene& s) {
  SpectralMoments m;
  m.reset(s.shape.bands);
  const std::size_t stride = bsq_plane_stride(s.shape);
  std::vector<float> px(s.shape.bands);
  for (std::size_t p = 0; p < s.shape.pixels(); ++p) {
    for (int b = 0; b < s.shape.bands; ++b) px[b] = s.host[b * stride + p];
    m.add(px.data());
  }
  return m;
}

void test_traits_are_consistent() {
  CHECK(traits_of(Detector::Sam).polarity == ScorePolarity::LowerIsBetter);
  for (Detector d : {Detector::Rx, Detector::Ace, Detector::Cem}) {
    CHECK(traits_of(d).polarity == ScorePolarity::HigherIsBetter);
    CHECK(traits_of(d).needs_statistics);
    Detector back;
    CHECK(parse_detector(to_string(d), &back) && back == d);
  }
  CHECK(!traits_of(Detector::Rx).needs_targets);
  Detector x;
  CHECK(!parse_detector("mahalanobis", &x));
}

void test_whitener_whitens_the_covariance() {
  const Scene s = make_scene(48, 64, 24, 2, 0.0f, 101);
  const SpectralMoments m = host_moments(s);
  DetectorStatistics st;
  std::string err;
  CHECK(build_statistics(m, s.library, 1e-6, &st, &err));
  CHECK(st.valid && st.bands == 24 && st.num_targets == 2);
  const int B = 24;
  const std::vector<double> S = m.covariance(1e-6);
  // W S W^T = I  (W lower triangular, upper exactly zero)
  double worst = 0.0;
  for (int i = 0; i < B; ++i) {
    for (int j = i + 1; j < B; ++j) CHECK(st.whitener[i * B + j] == 0.0f);
    for (int j = 0; j < B; ++j) {
      double v = 0.0;
      for (int k = 0; k < B; ++k)
        for (int l = 0; l < B; ++l) v += double(st.whitener[i * B + k]) * S[k * B + l] * st.whitener[j * B + l];
      worst = std::max(worst, std::fabs(v - (i == j ? 1.0 : 0.0)));
    }
  }
  CHECK(worst < 1e-3);  // float whitener, condition number of the scene
}

void test_cem_passes_its_target_at_unit_gain() {
  const Scene s = make_scene(40, 50, 16, 3, 0.0f, 202);
  DetectorStatistics st;
  std::string err;
  CHECK(build_statistics(host_moments(s), s.library, 1e-6, &st, &err));
  for (int t = 0; t < 3; ++t) {
    double g = 0.0;
    for (int b = 0; b < 16; ++b) g += double(st.cem_weight[t * 16 + b]) * s.library.targets[t].values[b];
    CHECK_CLOSE(g, 1.0, 1e-4);
  }
}

void test_singular_covariance_is_reported_not_silently_wrong() {
  // every pixel the same spectrum: the covariance is exactly zero
  SpectralMoments m;
  m.reset(4);
  const float x[4] = {0.2f, 0.4f, 0.6f, 0.8f};
  for (int i = 0; i < 50; ++i) m.add(x);
  SpectralLibrary lib;
  DetectorStatistics st;
  std::string err;
  CHECK(!build_statistics(m, lib, 0.0, &st, &err));
  CHECK(!st.valid);
  CHECK(err.find("loading") != std::string::npos);
  CHECK(build_statistics(m, lib, 1e-3, &st, &err));
  SpectralMoments empty;
  empty.reset(4);
  CHECK(!build_statistics(empty, lib, 1e-3, &st, &err));
}

void test_library_band_mismatch_is_rejected() {
  SpectralMoments m;
  m.reset(4);
  const float x[4] = {0.2f, 0.4f, 0.6f, 0.8f};
  m.add(x);
  SpectralLibrary lib;
  lib.targets.push_back({"t", {1.0f, 2.0f, 3.0f}, {}});
  DetectorStatistics st;
  std::string err;
  CHECK(!build_statistics(m, lib, 1e-3, &st, &err));
  CHECK(err.find("bands") != std::string::npos);
}

void test_device_statistics_match_host_moments() {
  const Scene s = make_scene(64, 96, 32, 4, 0.002f, 303);
  Dev<float> cube(s.host);
  DeviceStatistics ds;
  int status = -1;
  CHECK_CUDA(ds.build(cube.p, s.shape, false, s.library, 1e-6, nullptr, &status));
  CHECK(status == 0);
  DetectorStatistics dev, host;
  std::string err;
  CHECK(ds.download(&dev));
  CHECK(build_statistics(host_moments(s), s.library, 1e-6, &host, &err));
  double worst = 0.0, scale = 0.0;
  for (std::size_t i = 0; i < host.whitener.size(); ++i) {
    worst = std::max(worst, double(std::fabs(dev.whitener[i] - host.whitener[i])));
    scale = std::max(scale, double(std::fabs(host.whitener[i])));
  }
  CHECK(worst <= 1e-4 * scale);
}

void test_rx_ranks_anomalies_and_ace_stays_in_range() {
  const int H = 96, W = 128, B = 32, T = 4;
  const Scene s = make_scene(H, W, B, T, 0.004f, 404);
  Dev<float> cube(s.host);
  DeviceStatistics ds;
  CHECK_CUDA(ds.build(cube.p, s.shape, false, s.library, 1e-6, nullptr));
  const std::size_t P = s.shape.pixels();
  Dev<float> rx(P), ace(P), maps(T * P);
  Dev<std::int32_t> which(P);
  CHECK_CUDA(launch_rx_ace(cube.p, s.shape, false, ds, rx.p, ace.p, which.p, maps.p, P, nullptr));
  CHECK_CUDA(cudaDeviceSynchronize());
  const std::vector<float> r = rx.download(), a = ace.download(), m = maps.download();
  const std::vector<std::int32_t> w = which.download();
  double bg = 0.0, an = 0.0;
  int nbg = 0, nan_ = 0;
  for (std::size_t p = 0; p < P; ++p) {
    if (s.truth[p] == 0) {
      bg += r[p];
      ++nbg;
    } else if (s.truth[p] == 255) {
      an += r[p];
      ++nan_;
    }
    CHECK(a[p] >= 0.0f && a[p] <= 1.0f);
    // the best is the largest per-target map, lowest index on ties
    int best = -1;
    float bv = 0.0f;
    for (int t = 0; t < T; ++t)
      if (best < 0 || m[t * P + p] > bv) {
        best = t;
        bv = m[t * P + p];
      }
    CHECK(w[p] == best || (w[p] == -1 && bv == 0.0f));
  }
  CHECK(nan_ > 0);
  // RX of Gaussian-like background averages about the band count (chi-square mean)
  CHECK(bg / nbg > 0.5 * B && bg / nbg < 1.5 * B);
  CHECK(an / nan_ > 3.0 * (bg / nbg));
  // ACE peaks on implanted targets
  double on = 0.0;
  int non = 0;
  for (std::size_t p = 0; p < P; ++p)
    if (s.truth[p] >= 1 && s.truth[p] <= T) {
      on += a[p];
      ++non;
    }
  CHECK(non > 0 && on / non > 0.3);
}

void test_cem_is_near_unity_on_its_target() {
  const Scene s = make_scene(64, 64, 24, 3, 0.0f, 505);
  Dev<float> cube(s.host);
  DeviceStatistics ds;
  CHECK_CUDA(ds.build(cube.p, s.shape, false, s.library, 1e-6, nullptr));
  const std::size_t P = s.shape.pixels();
  Dev<float> best(P), maps(3 * P);
  Dev<std::int32_t> which(P);
  CHECK_CUDA(launch_cem(cube.p, s.shape, false, ds, best.p, which.p, maps.p, P, nullptr));
  CHECK_CUDA(cudaDeviceSynchronize());
  const std::vector<float> b = best.download();
  const std::vector<std::int32_t> w = which.download();
  double bg = 0.0, on = 0.0;
  int nbg = 0, non = 0, hits = 0;
  for (std::size_t p = 0; p < P; ++p) {
    if (s.truth[p] == 0) {
      bg += std::fabs(b[p]);
      ++nbg;
    } else if (s.truth[p] <= 3) {
      on += b[p];
      ++non;
      hits += w[p] == s.truth[p] - 1;
    }
  }
  CHECK(non > 0);
  CHECK(on / non > 5.0 * bg / nbg);
  CHECK(hits >= non * 8 / 10);
}

void test_stats_accumulators_match_host_moments() {
  const Scene s = make_scene(50, 70, 12, 0, 0.0f, 606);
  const int B = 12;
  Dev<float> cube(s.host);
  Dev<double> sum(B), outer(B * B);
  std::vector<float> ref(B, 0.25f);
  Dev<float> d_ref(ref);
  CHECK_CUDA(launch_reset_moments(sum.p, outer.p, B, nullptr));
  // two accumulations of the same cube: twice the sums
  CHECK_CUDA(launch_accumulate_moments(cube.p, s.shape, d_ref.p, sum.p, outer.p, nullptr));
  CHECK_CUDA(launch_accumulate_moments(cube.p, s.shape, d_ref.p, sum.p, outer.p, nullptr));
  SpectralMoments got;
  CHECK_CUDA(read_moments(sum.p, outer.p, B, 2.0 * s.shape.pixels(), ref.data(), &got));
  SpectralMoments want = host_moments(s);
  want.merge(host_moments(s));
  const std::vector<double> c0 = want.covariance(), c1 = got.covariance();
  double worst = 0.0, scale = 0.0;
  for (std::size_t i = 0; i < c0.size(); ++i) {
    worst = std::max(worst, std::fabs(c0[i] - c1[i]));
    scale = std::max(scale, std::fabs(c0[i]));
  }
  CHECK(worst < 1e-6 * scale);
  const std::vector<double> m0 = want.mean(), m1 = got.mean();
  for (int b = 0; b < B; ++b) CHECK_CLOSE(m1[b], m0[b], 1e-6 * std::fabs(m0[b]) + 1e-9);
  CHECK(moment_cube_reads(B) >= 1);
}

void test_chi_squared_threshold_matches_the_closed_form() {
  // two degrees of freedom: P(X > t) = exp(-t/2)
  for (double rate : {0.1, 1e-3, 1e-6}) CHECK_CLOSE(rx_threshold_for_false_alarm_rate(2, rate), -2.0 * std::log(rate), 1e-6);
  // larger B: the tail at the threshold equals the rate (monotone, above the mean)
  const double t = rx_threshold_for_false_alarm_rate(113, 1e-3);
  CHECK(t > 113.0 && t < 200.0);
  bool threw = false;
  try {
    rx_threshold_for_false_alarm_rate(0, 0.1);
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  CHECK(threw);
}

}  // namespace

int main() {
  test_traits_are_consistent();
  test_whitener_whitens_the_covariance();
  test_cem_passes_its_target_at_unit_gain();
  test_singular_covariance_is_reported_not_silently_wrong();
  test_library_band_mismatch_is_rejected();
  test_device_statistics_match_host_moments();
  test_rx_ranks_anomalies_and_ace_stays_in_range();
  test_cem_is_near_unity_on_its_target();
  test_stats_accumulators_match_host_moments();
  test_chi_squared_threshold_matches_the_closed_form();
  return tcheck::finish("detector_gpu");
}
