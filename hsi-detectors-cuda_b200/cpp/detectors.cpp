// hsi/detectors.hpp over the C ABI: device statistics, RX/ACE and CEM.
#include "hsi/detectors.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "hsi/sam_cuda.hpp"
#include "status.hpp"
#include "workspace.hpp"

namespace hsi {

using detail::as_stream;
using detail::to_cuda;

DeviceStatistics::~DeviceStatistics() { release(); }

void DeviceStatistics::release() {
  cudaFree(packed_);
  cudaFree(moments_);
  cudaFree(cem_);
  cudaFree(library_);
  cudaFree(workspace_);
  packed_ = moments_ = nullptr;
  cem_ = library_ = nullptr;
  workspace_ = nullptr;
  workspace_bytes_ = 0;
  bands_ = targets_ = 0;
}

cudaError_t DeviceStatistics::build(const void* d_cube, CubeShape shape, bool half, const SpectralLibrary& library,
                                    double diagonal_loading, cudaStream_t stream, int* status) {
  if (status) *status = HSI_OK;
  if (!d_cube || !shape.valid() || shape.bands > HSI_MAX_BANDS) return cudaErrorInvalidValue;
  const int B = shape.bands, T = library.size();
  if (T > 0 && library.bands() != B) return cudaErrorInvalidValue;
  const std::size_t ws = std::max(hsi_stats_workspace_bytes(shape.height, shape.width, B),
                                  hsi_factor_workspace_bytes(1, B));
  if (B != bands_ || T != targets_ || ws > workspace_bytes_) {
    release();
    cudaError_t e = cudaMalloc(&packed_, sizeof(double) * hsi_statistics_elements(B, T));
    if (e == cudaSuccess) e = cudaMalloc(&moments_, sizeof(double) * (B + static_cast<std::size_t>(B) * B + 1));
    if (e == cudaSuccess) e = cudaMalloc(&cem_, sizeof(float) * std::max(1, T * B));
    if (e == cudaSuccess) e = cudaMalloc(&library_, sizeof(float) * std::max(1, T * B) + 256);
    if (e == cudaSuccess) e = cudaMalloc(&workspace_, ws);
    if (e != cudaSuccess) {
      release();
      return e;
    }
    bands_ = B;
    targets_ = T;
    workspace_bytes_ = ws;
  }
  int* d_status = reinterpret_cast<int*>(library_ + std::max(1, T * B));
  cudaError_t e = cudaSuccess;
  if (T > 0) {
    const std::vector<float> flat = library.flatten();
    e = cudaMemcpyAsync(library_, flat.data(), sizeof(float) * flat.size(), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // `flat` goes out of scope
    if (e != cudaSuccess) return e;
  }
  int st = hsi_scene_moments(d_cube, shape.height, shape.width, B, half ? HSI_F16 : HSI_F32,
                             static_cast<int64_t>(bsq_plane_stride(shape)), moments_, nullptr, workspace_,
                             workspace_bytes_, as_stream(stream));
  if (st == HSI_OK)
    st = hsi_build_statistics(1, B, T, diagonal_loading, moments_, T > 0 ? library_ : nullptr, 0, packed_,
                              nullptr, T > 0 ? cem_ : nullptr, d_status, workspace_, workspace_bytes_,
                              as_stream(stream));
  if (st != HSI_OK) return to_cuda(st);
  int h_status = 0;
  e = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return e;
  if (status) *status = h_status;
  return h_status == HSI_OK ? cudaSuccess : cudaErrorInvalidValue;
}

bool DeviceStatistics::download(DetectorStatistics* out) const {
  if (!out || !packed_) return false;
  const std::size_t n = hsi_statistics_elements(bands_, targets_);
  std::vector<double> h(n);
  if (cudaMemcpy(h.data(), packed_, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
  const std::size_t B = static_cast<std::size_t>(bands_), T = static_cast<std::size_t>(targets_);
  const double* p = h.data();
  const auto take = [&](std::vector<float>& v, std::size_t k) {
    v.resize(k);
    for (std::size_t i = 0; i < k; ++i) v[i] = static_cast<float>(p[i]);
    p += k;
  };
  out->bands = bands_;
  out->num_targets = targets_;
  take(out->mean, B);
  take(out->whitener, B * B);
  take(out->target_white, T * B);
  take(out->target_norm2, T);
  take(out->cem_weight, T * B);
  out->valid = true;
  return true;
}

cudaError_t launch_rx_ace(const void* d_cube, CubeShape shape, bool half, const DeviceStatistics& stats,
                          float* d_rx, float* d_ace_best, std::int32_t* d_ace_target, float* d_ace_maps,
                          std::size_t map_stride, cudaStream_t stream) {
  if (!d_cube || !shape.valid() || shape.bands != stats.bands() || !stats.packed()) return cudaErrorInvalidValue;
  const int T = (d_ace_best || d_ace_target || d_ace_maps) ? stats.num_targets() : 0;
  // the tensor-core whitening holds up to 127 bands; wider cubes take the FP32 CUDA-core kernel
  const bool tensor = shape.bands <= 127;
  const std::size_t ws = tensor ? hsi_rx_ace_workspace_bytes(shape.bands, T)
                                : hsi_rx_ace_simt_workspace_bytes(shape.bands, T);
  void* scratch = nullptr;
  const cudaError_t e = detail::stream_scratch(stream, ws, &scratch);
  if (e != cudaSuccess) return e;
  const auto fn = tensor ? hsi_rx_ace : hsi_rx_ace_simt;
  return to_cuda(fn(d_cube, shape.height, shape.width, shape.bands, half ? HSI_F16 : HSI_F32,
                    static_cast<int64_t>(bsq_plane_stride(shape)), stats.packed(), T, d_rx, d_ace_best, d_ace_target,
                    d_ace_maps, static_cast<int64_t>(map_stride), scratch, ws, as_stream(stream)));
}

cudaError_t launch_cem(const void* d_cube, CubeShape shape, bool half, const DeviceStatistics& stats, float* d_best,
                       std::int32_t* d_target, float* d_maps, std::size_t map_stride, cudaStream_t stream) {
  if (!d_cube || !shape.valid() || shape.bands != stats.bands() || stats.num_targets() <= 0 || !stats.cem_weights())
    return cudaErrorInvalidValue;
  if (d_maps && map_stride < shape.pixels()) return cudaErrorInvalidValue;
  hsi_frame f;
  std::memset(&f, 0, sizeof(f));
  f.cube = d_cube;
  f.plane_stride = static_cast<int64_t>(bsq_plane_stride(shape));
  f.height = shape.height;
  f.width = shape.width;
  f.bands = shape.bands;
  f.dtype = half ? HSI_F16 : HSI_F32;
  f.num_cem = stats.num_targets();
  f.cem_weights = stats.cem_weights();
  f.cem_maps = d_maps;
  f.cem_best = d_best;
  f.cem_best_target = d_target;
  f.map_stride = static_cast<int64_t>(d_maps ? map_stride : shape.pixels());
  return to_cuda(hsi_score_frames(&f, 1, as_stream(stream)));
}

// ---- chi-square threshold ------------------------------------------------------
//
// P(a, x), the regularised lower incomplete gamma function: its power series
// for x < a + 1, else 1 - Q(a, x) with Q from the continued fraction
// evaluated by the modified Lentz method (both standard; e.g. Press et al.,
// Numerical Recipes, 6.2).  The threshold t solves P(B/2, t/2) = 1 - rate by
// bisection, as the reference does (src/detectors_cpu.cpp:189-206).
namespace {

double lower_gamma_regularised(double a, double x) {
  if (x <= 0.0) return 0.0;
  const double log_prefix = -x + a * std::log(x) - std::lgamma(a);
  if (x < a + 1.0) {
    double term = 1.0 / a, sum = term;
    for (int n = 1; n < 100000; ++n) {
      term *= x / (a + n);
      sum += term;
      if (std::fabs(term) < std::fabs(sum) * 1e-17) break;
    }
    return sum * std::exp(log_prefix);
  }
  const double tiny = 1e-300;
  double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
  for (int i = 1; i < 100000; ++i) {
    const double an = -i * (i - a);
    b += 2.0;
    d = an * d + b;
    if (std::fabs(d) < tiny) d = tiny;
    c = b + an / c;
    if (std::fabs(c) < tiny) c = tiny;
    d = 1.0 / d;
    const double delta = d * c;
    h *= delta;
    if (std::fabs(delta - 1.0) < 1e-17) break;
  }
  return 1.0 - std::exp(log_prefix) * h;
}

}  // namespace

double rx_threshold_for_false_alarm_rate(int bands, double rate) {
  if (bands <= 0) throw std::invalid_argument("rx_threshold_for_false_alarm_rate: bands must be positive");
  if (!(rate > 0.0 && rate < 1.0))
    throw std::invalid_argument("rx_threshold_for_false_alarm_rate: rate must lie in (0, 1)");
  const double a = 0.5 * bands, want = 1.0 - rate;
  double lo = 0.0, hi = std::max(16.0, 4.0 * bands);
  while (lower_gamma_regularised(a, 0.5 * hi) < want && hi < 1e9) hi *= 2.0;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    (lower_gamma_regularised(a, 0.5 * mid) < want ? lo : hi) = mid;
  }
  return 0.5 * (lo + hi);
}

}  // namespace hsi
