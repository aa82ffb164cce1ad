// The spectral-angle and detection properties of the reference's SAM tests,
// checked through the drop-in GPU API (hsi::launch_sam_best,
// hsi::launch_sam_maps, hsi::launch_detect) on the device.
#include <algorithm>
#include <cstdint>
#include <random>
#include <vector>

#include "check.hpp"
#include "hsi/detect_cuda.hpp"
#include "hsi/sam_cuda.hpp"

using namespace hsi;
using tcheck::Dev;

namespace {

constexpr float kHalfPi = 1.57079632679489661923f;

CubeShape shape_of(int h, int w, int b) {
  CubeShape s;
  s.height = h;
  s.width = w;
  s.bands = b;
  return s;
}

// Packed host BSQ -> device cube at bsq_plane_stride.
Dev<float>* to_device(const std::vector<float>& packed, CubeShape s) {
  auto* d = new Dev<float>(bsq_device_elements(s));
  const std::size_t P = s.pixels(), stride = bsq_plane_stride(s);
  for (int b = 0; b < s.bands; ++b)
    cudaMemcpy(d->p + b * stride, packed.data() + b * P, sizeof(float) * P, cudaMemcpyHostToDevice);
  return d;
}

struct Best {
  std::vector<float> angle;
  std::vector<std::int32_t> which;
};

Best sam_best(const std::vector<float>& packed, CubeShape s, const SpectralLibrary& lib,
              SamVariant v = SamVariant::Optimized) {
  const std::vector<float> flat = lib.flatten(), norms = lib.norms();
  CHECK_CUDA(upload_targets(flat.data(), norms.data(), lib.size(), lib.bands()));
  Dev<float> t(flat), n(norms), score(s.pixels());
  Dev<std::int32_t> which(s.pixels());
  Dev<float>* cube = to_device(packed, s);
  CHECK_CUDA(launch_sam_best(v, cube->p, s, t.p, n.p, lib.size(), score.p, which.p, nullptr));
  CHECK_CUDA(cudaDeviceSynchronize());
  delete cube;
  return {score.download(), which.download()};
}

std::vector<Detection> detect(const std::vector<float>& score, const std::vector<std::int32_t>& which, CubeShape s,
                              DetectionParams p) {
  Dev<float> d_score(score);
  Dev<std::int32_t> d_which(which);
  Dev<Detection> out(static_cast<std::size_t>(p.max_detections));
  Dev<unsigned> count(1);
  CHECK_CUDA(launch_detect(d_score.p, d_which.p, s, p, out.p, count.p, nullptr));
  CHECK_CUDA(cudaDeviceSynchronize());
  const unsigned n = count.download()[0];
  std::vector<Detection> all = out.download();
  all.resize(std::min<std::size_t>(n, all.size()));
  return all;
}

void test_identical_spectrum_is_zero_angle() {
  const CubeShape s = shape_of(1, 1, 8);
  std::vector<float> target{0.1f, 0.4f, 0.9f, 0.3f, 0.2f, 0.7f, 0.5f, 0.6f};
  SpectralLibrary lib;
  lib.targets.push_back({"t", target, {}});
  const Best r = sam_best(target, s, lib);
  CHECK_CLOSE(r.angle[0], 0.0, 1e-3);  // acos near 1 amplifies FP32 rounding of the cosine
  CHECK(r.which[0] == 0);
}

void test_scale_invariance() {
  const int B = 16;
  const CubeShape s = shape_of(1, 5, B);
  std::mt19937 rng(7);
  std::uniform_real_distribution<float> u(0.05f, 1.0f);
  std::vector<float> target(B), pixel(B);
  for (int b = 0; b < B; ++b) {
    target[b] = u(rng);
    pixel[b] = u(rng);
  }
  const float gains[5] = {1.0f, 0.01f, 0.5f, 3.0f, 250.0f};
  std::vector<float> cube(s.elements());
  for (int b = 0; b < B; ++b)
    for (int p = 0; p < 5; ++p) cube[b * 5 + p] = pixel[b] * gains[p];
  SpectralLibrary lib;
  lib.targets.push_back({"t", target, {}});
  const Best r = sam_best(cube, s, lib);
  for (int p = 1; p < 5; ++p) CHECK_CLOSE(r.angle[p], r.angle[0], 1e-4);
}

void test_orthogonal_and_zero_pixels() {
  const CubeShape s = shape_of(1, 2, 4);
  std::vector<float> cube(s.elements(), 0.0f);
  const float v[4] = {0.0f, 1.0f, 0.0f, 1.0f};
  for (int b = 0; b < 4; ++b) cube[b * 2] = v[b];
  SpectralLibrary lib;
  lib.targets.push_back({"t", {1.0f, 0.0f, 1.0f, 0.0f}, {}});
  const Best r = sam_best(cube, s, lib);
  CHECK_CLOSE(r.angle[0], kHalfPi, 1e-5);
  CHECK_CLOSE(r.angle[1], kHalfPi, 1e-5);  // no direction: the maximum angle, never NaN
  CHECK(!std::isnan(r.angle[1]));
}

void test_best_match_picks_the_nearest_target() {
  const CubeShape s = shape_of(1, 1, 6);
  std::vector<float> pixel{0.1f, 0.2f, 0.3f, 0.4f, 0.5f, 0.6f};
  SpectralLibrary lib;
  lib.targets.push_back({"far", {1, 0, 0, 0, 0, 0}, {}});
  lib.targets.push_back({"near", {0.2f, 0.4f, 0.6f, 0.8f, 1.0f, 1.2f}, {}});
  lib.targets.push_back({"middling", {0.6f, 0.5f, 0.4f, 0.3f, 0.2f, 0.1f}, {}});
  const Best r = sam_best(pixel, s, lib);
  CHECK(r.which[0] == 1);
  CHECK_CLOSE(r.angle[0], 0.0, 1e-3);
  // the per-target maps agree with the best-match reduction
  const std::vector<float> flat = lib.flatten(), norms = lib.norms();
  Dev<float> t(flat), n(norms), maps(3);
  Dev<float>* cube = to_device(pixel, s);
  CHECK_CUDA(launch_sam_maps(cube->p, s, false, t.p, n.p, 3, maps.p, 1, nullptr));
  CHECK_CUDA(cudaDeviceSynchronize());
  delete cube;
  const std::vector<float> all = maps.download();
  CHECK_CLOSE(all[1], r.angle[0], 1e-6);
  CHECK(all[0] > r.angle[0] && all[2] > r.angle[0]);
}

void test_variants_agree() {
  // Optimized (fp32 BSQ), Half (fp16 BSQ) and BipDirect (fp32 BIP) on one cube
  const CubeShape s = shape_of(37, 53, 24);
  std::mt19937 rng(11);
  std::uniform_real_distribution<float> u(0.0f, 1.0f);
  std::vector<float> cube(s.elements());
  for (float& x : cube) x = u(rng);
  SpectralLibrary lib;
  for (int t = 0; t < 5; ++t) {
    std::vector<float> v(s.bands);
    for (float& x : v) x = u(rng);
    lib.targets.push_back({"t" + std::to_string(t), v, {}});
  }
  const Best a = sam_best(cube, s, lib, SamVariant::Optimized);
  const Best base = sam_best(cube, s, lib, SamVariant::Baseline);
  // fp16 cube, narrowed on the device
  const std::vector<float> flat = lib.flatten(), norms = lib.norms();
  Dev<float> t(flat), n(norms), score(s.pixels());
  Dev<std::int32_t> which(s.pixels());
  Dev<float>* d32 = to_device(cube, s);
  Dev<std::uint16_t> d16(bsq_device_elements(s));
  CHECK_CUDA(launch_narrow_to_half(d32->p, d16.p, bsq_device_elements(s), nullptr));
  CHECK_CUDA(launch_sam_best(SamVariant::Half, d16.p, s, t.p, n.p, 5, score.p, which.p, nullptr));
  CHECK_CUDA(cudaDeviceSynchronize());
  const std::vector<float> half = score.download();
  // BIP layout on the host, transposed on the device
  std::vector<float> bip(s.elements());
  for (int b = 0; b < s.bands; ++b)
    for (std::size_t p = 0; p < s.pixels(); ++p) bip[p * s.bands + b] = cube[b * s.pixels() + p];
  Dev<float> d_bip(bip);
  CHECK_CUDA(launch_sam_best(SamVariant::BipDirect, d_bip.p, s, t.p, n.p, 5, score.p, which.p, nullptr));
  CHECK_CUDA(cudaDeviceSynchronize());
  const std::vector<float> from_bip = score.download();
  const std::vector<std::int32_t> which_bip = which.download();
  delete d32;
  double worst_half = 0.0;
  for (std::size_t p = 0; p < s.pixels(); ++p) {
    CHECK(a.angle[p] == base.angle[p]);
    CHECK(a.angle[p] == from_bip[p]);
    CHECK(a.which[p] == which_bip[p]);
    worst_half = std::max(worst_half, static_cast<double>(std::fabs(a.angle[p] - half[p])));
  }
  CHECK(worst_half < 5e-3);  // fp16 storage of the cube: ~1e-3 rad
}

void test_nms_keeps_one_pixel_per_blob() {
  const CubeShape s = shape_of(9, 9, 1);
  std::vector<float> angle(81, 1.0f);
  std::vector<std::int32_t> which(81, 0);
  for (int y = 3; y <= 5; ++y)
    for (int x = 3; x <= 5; ++x) angle[y * 9 + x] = 0.05f;
  angle[4 * 9 + 4] = 0.01f;
  DetectionParams p;
  p.threshold = 0.1f;
  p.nms_radius = 0;
  CHECK(detect(angle, which, s, p).size() == 9);
  p.nms_radius = 2;
  const std::vector<Detection> peaks = detect(angle, which, s, p);
  CHECK(peaks.size() == 1);
  if (peaks.size() == 1) {
    CHECK(peaks[0].x == 4 && peaks[0].y == 4);
    CHECK_CLOSE(peaks[0].score, 0.01, 1e-6);
  }
}

void test_nms_breaks_ties_by_index() {
  const CubeShape s = shape_of(5, 5, 1);
  std::vector<float> angle(25, 1.0f);
  std::vector<std::int32_t> which(25, 0);
  for (int y = 1; y <= 2; ++y)
    for (int x = 1; x <= 2; ++x) angle[y * 5 + x] = 0.02f;
  DetectionParams p;
  p.threshold = 0.1f;
  p.nms_radius = 2;
  const std::vector<Detection> peaks = detect(angle, which, s, p);
  CHECK(peaks.size() == 1);
  if (peaks.size() == 1) CHECK(peaks[0].x == 1 && peaks[0].y == 1);
}

void test_polarity_inverts_the_detector() {
  const CubeShape s = shape_of(7, 7, 1);
  std::vector<float> score(49, 0.5f);
  std::vector<std::int32_t> which(49, 0);
  score[2 * 7 + 2] = 0.01f;
  score[5 * 7 + 5] = 0.99f;
  DetectionParams p;
  p.nms_radius = 1;
  p.threshold = 0.1f;
  p.polarity = ScorePolarity::LowerIsBetter;
  const std::vector<Detection> low = detect(score, which, s, p);
  CHECK(low.size() == 1);
  if (low.size() == 1) CHECK(low[0].x == 2 && low[0].y == 2);
  p.threshold = 0.9f;
  p.polarity = ScorePolarity::HigherIsBetter;
  const std::vector<Detection> high = detect(score, which, s, p);
  CHECK(high.size() == 1);
  if (high.size() == 1) CHECK(high[0].x == 5 && high[0].y == 5);
}

void test_polarity_picks_the_right_extremum_in_a_blob() {
  const CubeShape s = shape_of(9, 9, 1);
  std::vector<float> score(81, 0.5f);
  std::vector<std::int32_t> which(81, 0);
  for (int y = 3; y <= 5; ++y)
    for (int x = 3; x <= 5; ++x) score[y * 9 + x] = 0.8f;
  score[3 * 9 + 3] = 0.6f;
  score[5 * 9 + 5] = 0.95f;
  DetectionParams p;
  p.nms_radius = 3;
  p.threshold = 0.55f;
  p.polarity = ScorePolarity::HigherIsBetter;
  const std::vector<Detection> found = detect(score, which, s, p);
  CHECK(found.size() == 1);
  if (found.size() == 1) {
    CHECK(found[0].x == 5 && found[0].y == 5);
    CHECK_CLOSE(found[0].score, 0.95, 1e-6);
  }
}

void test_capacity_counts_everything_but_writes_the_first() {
  const CubeShape s = shape_of(10, 10, 1);
  std::vector<float> score(100, 0.0f);
  std::vector<std::int32_t> which(100, 3);
  DetectionParams p;
  p.threshold = 0.5f;
  p.nms_radius = 0;
  p.max_detections = 7;
  Dev<float> d_score(score);
  Dev<std::int32_t> d_which(which);
  Dev<Detection> out(7);
  Dev<unsigned> count(1);
  CHECK_CUDA(launch_detect(d_score.p, d_which.p, s, p, out.p, count.p, nullptr));
  CHECK_CUDA(cudaDeviceSynchronize());
  CHECK(count.download()[0] == 100);
  const std::vector<Detection> d = out.download();
  for (int i = 0; i < 7; ++i) CHECK(d[i].x == i && d[i].y == 0 && d[i].target == 3);
}

void test_invalid_arguments_are_rejected() {
  const CubeShape bad = shape_of(0, 4, 4);
  Dev<float> buf(64);
  Dev<std::int32_t> ibuf(64);
  CHECK(launch_sam_best(SamVariant::Optimized, buf.p, bad, buf.p, buf.p, 1, buf.p, ibuf.p, nullptr) ==
        cudaErrorInvalidValue);
  CHECK(upload_targets(buf.p, buf.p, 0, 4) == cudaErrorInvalidValue);
  DetectionParams p;
  CHECK(launch_detect(buf.p, ibuf.p, bad, p, nullptr, nullptr, nullptr) == cudaErrorInvalidValue);
  SamVariant v;
  CHECK(parse_sam_variant("half", &v) && v == SamVariant::Half);
  CHECK(!parse_sam_variant("nonsense", &v));
}

}  // namespace

int main() {
  test_identical_spectrum_is_zero_angle();
  test_scale_invariance();
  test_orthogonal_and_zero_pixels();
  test_best_match_picks_the_nearest_target();
  test_variants_agree();
  test_nms_keeps_one_pixel_per_blob();
  test_nms_breaks_ties_by_index();
  test_polarity_inverts_the_detector();
  test_polarity_picks_the_right_extremum_in_a_blob();
  test_capacity_counts_everything_but_writes_the_first();
  test_invalid_arguments_are_rejected();
  return tcheck::finish("sam_gpu");
}
