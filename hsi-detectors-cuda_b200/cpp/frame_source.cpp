// make_synthetic_source: frames of the library's scene model, generated on
// the device (hsi_generate) and copied into the caller's host buffer.
#include <cuda_runtime.h>

#include <cstring>
#include <sstream>
#include <stdexcept>

#include "hsi/frame_source.hpp"
#include "hsi_b200.h"

namespace hsi {
namespace {

class SyntheticSource final : public FrameSource {
 public:
  explicit SyntheticSource(const SyntheticOptions& o) : opt_(o) {
    if (!o.shape.valid() || o.shape.bands > HSI_MAX_BANDS)
      throw std::invalid_argument("make_synthetic_source: invalid shape");
    if (o.background_endmembers < 1 || o.background_endmembers > 8)
      throw std::invalid_argument("make_synthetic_source: background_endmembers must be 1..8");
    if (o.num_targets < 0 || o.num_targets > 64)
      throw std::invalid_argument("make_synthetic_source: num_targets must be 0..64");
    scene_.bands = o.shape.bands;
    scene_.n_end = o.background_endmembers;
    scene_.n_targets = o.num_targets;
    scene_.target_frac = o.target_fraction;
    scene_.anomaly_frac = o.anomaly_fraction;
    scene_.noise_sigma = o.noise_sigma;
    scene_.library_seed = o.seed;
    scene_.frame_seed = o.seed + 1;
    const int n = o.background_endmembers + o.num_targets + 1;
    spectra_.resize(static_cast<std::size_t>(n) * o.shape.bands);
    if (hsi_scene_spectra(&scene_, spectra_.data()) != HSI_OK)
      throw std::runtime_error("make_synthetic_source: scene spectra");
    for (int t = 0; t < o.num_targets; ++t) {
      Spectrum s;
      s.name = "target" + std::to_string(t);
      const float* v = spectra_.data() + static_cast<std::size_t>(o.background_endmembers + t) * o.shape.bands;
      s.values.assign(v, v + o.shape.bands);
      library_.targets.push_back(std::move(s));
    }
    truth_.resize(o.shape.pixels());
  }

  ~SyntheticSource() override {
    cudaFree(d_cube_);
    cudaFree(d_spectra_);
    cudaFree(d_truth_);
  }

  CubeShape shape() const override { return opt_.shape; }
  Interleave interleave() const override { return Interleave::Bsq; }
  std::uint64_t length() const override { return opt_.length; }

  bool read_into(float* dst, std::size_t plane_stride, FrameMeta* meta) override {
    if (opt_.length && next_ >= opt_.length) return false;
    const CubeShape s = opt_.shape;
    const std::size_t P = s.pixels();
    if (plane_stride < P) throw std::invalid_argument("SyntheticSource::read_into: plane stride below pixels");
    if (!d_cube_ || plane_stride != stride_) {
      cudaFree(d_cube_);
      d_cube_ = nullptr;
      if (cudaMalloc(&d_cube_, sizeof(float) * plane_stride * s.bands) != cudaSuccess)
        throw std::runtime_error("SyntheticSource: device allocation failed");
      stride_ = plane_stride;
    }
    if (!d_spectra_) {
      if (cudaMalloc(&d_spectra_, sizeof(float) * spectra_.size()) != cudaSuccess ||
          cudaMalloc(&d_truth_, P) != cudaSuccess)
        throw std::runtime_error("SyntheticSource: device allocation failed");
      cudaMemcpy(d_spectra_, spectra_.data(), sizeof(float) * spectra_.size(), cudaMemcpyHostToDevice);
    }
    hsi_scene sc = scene_;
    sc.frame_seed = opt_.seed + 1 + next_;
    int st = hsi_generate(&sc, d_spectra_, s.height, s.width, 0, d_cube_, HSI_F32,
                          static_cast<int64_t>(plane_stride), d_truth_, nullptr);
    if (st != HSI_OK) throw std::runtime_error(std::string("SyntheticSource: ") + hsi_status_string(st));
    if (cudaMemcpy(dst, d_cube_, sizeof(float) * plane_stride * s.bands, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(truth_.data(), d_truth_, P, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw std::runtime_error("SyntheticSource: copy failed");
    if (meta) {
      meta->index = next_;
      meta->timestamp_s = static_cast<double>(next_) / 30.0;
    }
    ++next_;
    return true;
  }

  void reset() override { next_ = 0; }

  std::string describe() const override {
    std::ostringstream o;
    o << "synthetic " << opt_.shape.height << "x" << opt_.shape.width << "x" << opt_.shape.bands << ", "
      << opt_.background_endmembers << " endmembers, " << opt_.num_targets << " targets at " << opt_.target_fraction
      << " each, noise " << opt_.noise_sigma << ", seed " << opt_.seed;
    return o.str();
  }

  const std::uint8_t* truth_mask() const override { return truth_.data(); }
  const SpectralLibrary* library() const override { return &library_; }

 private:
  SyntheticOptions opt_;
  hsi_scene scene_{};
  std::vector<float> spectra_;
  SpectralLibrary library_;
  std::vector<std::uint8_t> truth_;
  std::uint64_t next_ = 0;
  void* d_cube_ = nullptr;
  float* d_spectra_ = nullptr;
  std::uint8_t* d_truth_ = nullptr;
  std::size_t stride_ = 0;
};

}  // namespace

std::unique_ptr<FrameSource> make_synthetic_source(const SyntheticOptions& options) {
  return std::unique_ptr<FrameSource>(new SyntheticSource(options));
}

}  // namespace hsi
