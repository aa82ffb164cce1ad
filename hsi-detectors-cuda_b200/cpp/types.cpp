// Host utilities of hsi/types.hpp and hsi/linalg.hpp.
#include <cmath>
#include <stdexcept>

#include "hsi/linalg.hpp"
#include "hsi/types.hpp"

namespace hsi {

const char* to_string(Interleave interleave) {
  switch (interleave) {
    case Interleave::Bsq: return "bsq";
    case Interleave::Bil: return "bil";
    case Interleave::Bip: return "bip";
  }
  return "unknown";
}

const char* to_string(ScorePolarity polarity) {
  return polarity == ScorePolarity::HigherIsBetter ? "higher-is-better" : "lower-is-better";
}

std::size_t HsiFrame::offset(int band, int y, int x) const {
  const std::size_t W = static_cast<std::size_t>(shape.width), H = static_cast<std::size_t>(shape.height);
  const std::size_t B = static_cast<std::size_t>(shape.bands);
  const std::size_t b = static_cast<std::size_t>(band), yy = static_cast<std::size_t>(y);
  const std::size_t xx = static_cast<std::size_t>(x);
  switch (interleave) {
    case Interleave::Bsq: return (b * H + yy) * W + xx;
    case Interleave::Bil: return (yy * B + b) * W + xx;
    case Interleave::Bip: return (yy * W + xx) * B + b;
  }
  return 0;
}

std::vector<float> SpectralLibrary::flatten() const {
  const int B = bands();
  std::vector<float> out;
  out.reserve(static_cast<std::size_t>(size()) * static_cast<std::size_t>(B));
  for (const Spectrum& t : targets) {
    if (t.bands() != B) throw std::invalid_argument("SpectralLibrary: targets differ in band count");
    out.insert(out.end(), t.values.begin(), t.values.end());
  }
  return out;
}

std::vector<float> SpectralLibrary::norms() const {
  std::vector<float> out;
  out.reserve(targets.size());
  for (const Spectrum& t : targets) {
    double s = 0.0;
    for (float v : t.values) s += static_cast<double>(v) * v;
    out.push_back(static_cast<float>(std::sqrt(s)));
  }
  return out;
}

void convert_interleave(const float* src, float* dst, CubeShape shape, Interleave from, Interleave to) {
  if (src == dst) throw std::invalid_argument("convert_interleave: src and dst alias");
  HsiFrame a, b;
  a.shape = b.shape = shape;
  a.interleave = from;
  b.interleave = to;
  for (int band = 0; band < shape.bands; ++band)
    for (int y = 0; y < shape.height; ++y)
      for (int x = 0; x < shape.width; ++x) dst[b.offset(band, y, x)] = src[a.offset(band, y, x)];
}

void convert_frame(HsiFrame& frame, Interleave to) {
  if (frame.interleave == to) return;
  std::vector<float> out(frame.data.size());
  convert_interleave(frame.data.data(), out.data(), frame.shape, frame.interleave, to);
  frame.data.swap(out);
  frame.interleave = to;
}

void SpectralMoments::reset(int n) {
  bands = n;
  count = 0.0;
  sum.assign(static_cast<std::size_t>(n), 0.0);
  sum_outer.assign(static_cast<std::size_t>(n) * static_cast<std::size_t>(n), 0.0);
}

void SpectralMoments::add(const float* spectrum) {
  for (int i = 0; i < bands; ++i) {
    const double xi = spectrum[i];
    sum[i] += xi;
    for (int j = 0; j < bands; ++j) sum_outer[static_cast<std::size_t>(i) * bands + j] += xi * spectrum[j];
  }
  count += 1.0;
}

void SpectralMoments::merge(const SpectralMoments& other) {
  if (other.empty()) return;
  if (empty() && bands != other.bands) {
    *this = other;
    return;
  }
  if (bands != other.bands) throw std::invalid_argument("SpectralMoments::merge: band counts differ");
  for (std::size_t i = 0; i < sum.size(); ++i) sum[i] += other.sum[i];
  for (std::size_t i = 0; i < sum_outer.size(); ++i) sum_outer[i] += other.sum_outer[i];
  count += other.count;
}

std::vector<double> SpectralMoments::mean() const {
  std::vector<double> m(static_cast<std::size_t>(bands), 0.0);
  if (count > 0.0)
    for (int i = 0; i < bands; ++i) m[i] = sum[i] / count;
  return m;
}

std::vector<double> SpectralMoments::covariance(double loading) const {
  const std::vector<double> m = mean();
  std::vector<double> c(sum_outer.size(), 0.0);
  for (int i = 0; i < bands; ++i)
    for (int j = 0; j < bands; ++j) {
      const std::size_t k = static_cast<std::size_t>(i) * bands + j;
      c[k] = (count > 0.0 ? sum_outer[k] / count : 0.0) - m[i] * m[j] + (i == j ? loading : 0.0);
    }
  return c;
}

std::vector<double> SpectralMoments::correlation(double loading) const {
  std::vector<double> r(sum_outer.size(), 0.0);
  for (int i = 0; i < bands; ++i)
    for (int j = 0; j < bands; ++j) {
      const std::size_t k = static_cast<std::size_t>(i) * bands + j;
      r[k] = (count > 0.0 ? sum_outer[k] / count : 0.0) + (i == j ? loading : 0.0);
    }
  return r;
}

void moments_from_shifted(const double* s1, const double* s2_lower, double count, const double* reference,
                          int bands, SpectralMoments* out) {
  out->reset(bands);
  out->count = count;
  for (int i = 0; i < bands; ++i) {
    const double ri = reference ? reference[i] : 0.0;
    out->sum[i] = s1[i] + count * ri;
  }
  for (int i = 0; i < bands; ++i) {
    const double ri = reference ? reference[i] : 0.0;
    for (int j = 0; j <= i; ++j) {
      const double rj = reference ? reference[j] : 0.0;
      // sum x_i x_j = S2_ij + r_i S1_j + S1_i r_j + N r_i r_j
      const double v = s2_lower[static_cast<std::size_t>(i) * bands + j] + ri * s1[j] + s1[i] * rj + count * ri * rj;
      out->sum_outer[static_cast<std::size_t>(i) * bands + j] = v;
      out->sum_outer[static_cast<std::size_t>(j) * bands + i] = v;
    }
  }
}

}  // namespace hsi
