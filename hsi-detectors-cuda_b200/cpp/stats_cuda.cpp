// hsi/stats_cuda.hpp and hsi/detector.hpp over the C ABI.
#include "hsi/stats_cuda.hpp"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hsi/detector.hpp"
#include "hsi/sam_cuda.hpp"
#include "status.hpp"
#include "workspace.hpp"

namespace hsi {

using detail::as_stream;
using detail::to_cuda;

cudaError_t launch_reset_moments(double* d_sum, double* d_sum_outer, int bands, cudaStream_t stream) {
  if (!d_sum || !d_sum_outer || bands <= 0) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(d_sum, 0, sizeof(double) * bands, stream);
  if (e != cudaSuccess) return e;
  return cudaMemsetAsync(d_sum_outer, 0, sizeof(double) * moment_outer_elements(bands), stream);
}

namespace {

// Moments of one cube into stream-ordered scratch, then the sums about
// `d_reference` added into the accumulators (d_outer may be scratch too).
cudaError_t accumulate(const float* d_cube, CubeShape shape, const float* d_reference, double* d_sum,
                       double* d_outer, cudaStream_t stream) {
  if (!d_cube || !shape.valid() || !d_sum || shape.bands > HSI_MAX_BANDS) return cudaErrorInvalidValue;
  const int B = shape.bands;
  const std::size_t ws_bytes = hsi_stats_workspace_bytes(shape.height, shape.width, B);
  const std::size_t m_bytes = sizeof(double) * (B + moment_outer_elements(B) + 1);
  const std::size_t o_bytes = d_outer ? 0 : sizeof(double) * moment_outer_elements(B);
  char* scratch = nullptr;
  const cudaError_t e =
      detail::stream_scratch(stream, ws_bytes + m_bytes + o_bytes, reinterpret_cast<void**>(&scratch));
  if (e != cudaSuccess) return e;
  double* moments = reinterpret_cast<double*>(scratch + ws_bytes);
  double* outer = d_outer ? d_outer : reinterpret_cast<double*>(scratch + ws_bytes + m_bytes);
  int st = hsi_scene_moments(d_cube, shape.height, shape.width, B, HSI_F32,
                             static_cast<int64_t>(bsq_plane_stride(shape)), moments, d_reference, scratch, ws_bytes,
                             as_stream(stream));
  if (st == HSI_OK) st = hsi_accumulate_shifted_moments(moments, d_reference, B, d_sum, outer, as_stream(stream));
  return to_cuda(st);
}

}  // namespace

cudaError_t launch_accumulate_mean(const float* d_cube_bsq, CubeShape shape, double* d_sum, cudaStream_t stream) {
  return accumulate(d_cube_bsq, shape, nullptr, d_sum, nullptr, stream);
}

cudaError_t launch_accumulate_moments(const float* d_cube_bsq, CubeShape shape, const float* d_reference,
                                      double* d_sum, double* d_sum_outer, cudaStream_t stream) {
  if (!d_sum_outer) return cudaErrorInvalidValue;
  return accumulate(d_cube_bsq, shape, d_reference, d_sum, d_sum_outer, stream);
}

cudaError_t read_moments(const double* d_sum, const double* d_sum_outer, int bands, double count,
                         const float* reference, SpectralMoments* out) {
  if (!d_sum || !d_sum_outer || bands <= 0 || !out) return cudaErrorInvalidValue;
  std::vector<double> s1(static_cast<std::size_t>(bands)), s2(moment_outer_elements(bands));
  cudaError_t e = cudaMemcpy(s1.data(), d_sum, sizeof(double) * s1.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(s2.data(), d_sum_outer, sizeof(double) * s2.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  std::vector<double> r;
  if (reference) r.assign(reference, reference + bands);
  moments_from_shifted(s1.data(), s2.data(), count, reference ? r.data() : nullptr, bands, out);
  return cudaSuccess;
}

int moment_cube_reads(int /*bands*/) { return 1; }

// ---- detector.hpp ------------------------------------------------------------

DetectorTraits traits_of(Detector detector) {
  switch (detector) {
    case Detector::Sam: return {"sam", true, false, ScorePolarity::LowerIsBetter, false};
    case Detector::Rx: return {"rx", false, true, ScorePolarity::HigherIsBetter, true};
    case Detector::Ace: return {"ace", true, true, ScorePolarity::HigherIsBetter, true};
    case Detector::Cem: return {"cem", true, true, ScorePolarity::HigherIsBetter, false};
  }
  return {"unknown", false, false, ScorePolarity::LowerIsBetter, false};
}

const char* to_string(Detector detector) { return traits_of(detector).name; }

bool parse_detector(const std::string& name, Detector* out) {
  for (Detector d : {Detector::Sam, Detector::Rx, Detector::Ace, Detector::Cem}) {
    if (name == traits_of(d).name) {
      *out = d;
      return true;
    }
  }
  return false;
}

namespace {

// Unpack hsi_build_statistics' packed layout (mean | whitener | target_white |
// target_norm2 | cem_weight) into the float DetectorStatistics.
template <typename T>
void unpack(const T* p, int B, int T_, DetectorStatistics* out) {
  const std::size_t b = static_cast<std::size_t>(B), t = static_cast<std::size_t>(T_);
  out->bands = B;
  out->num_targets = T_;
  out->mean.assign(p, p + b);
  p += b;
  out->whitener.assign(p, p + b * b);
  p += b * b;
  out->target_white.assign(p, p + t * b);
  p += t * b;
  out->target_norm2.assign(p, p + t);
  p += t;
  out->cem_weight.assign(p, p + t * b);
}

std::string loading_text(double loading) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%g", loading);
  return buf;
}

}  // namespace

bool build_statistics(const SpectralMoments& moments, const SpectralLibrary& library, double diagonal_loading,
                      DetectorStatistics* out, std::string* error) {
  const auto fail = [&](const std::string& message) {
    if (error) *error = message;
    if (out) out->valid = false;
    return false;
  };
  if (!out) return false;
  if (moments.empty()) return fail("no scene statistics accumulated yet");
  const int B = moments.bands;
  const int T = library.size();
  if (B <= 0 || B > HSI_MAX_BANDS) return fail("statistics cover " + std::to_string(B) + " bands; 1.." +
                                              std::to_string(HSI_MAX_BANDS) + " are supported");
  if (T > 0 && library.bands() != B)
    return fail("library has " + std::to_string(library.bands()) + " bands, statistics have " + std::to_string(B));

  std::vector<double> m(static_cast<std::size_t>(B) + moment_outer_elements(B) + 1);
  std::memcpy(m.data(), moments.sum.data(), sizeof(double) * B);
  std::memcpy(m.data() + B, moments.sum_outer.data(), sizeof(double) * moment_outer_elements(B));
  m.back() = moments.count;
  const std::vector<float> lib = library.flatten();
  const std::size_t n32 = hsi_statistics_elements(B, T);
  const std::size_t ws_bytes = hsi_factor_workspace_bytes(1, B);

  const std::size_t bytes_m = sizeof(double) * m.size(), bytes_lib = sizeof(float) * lib.size();
  const std::size_t bytes_out = sizeof(float) * n32;
  char* d = nullptr;
  const std::size_t total = bytes_m + bytes_lib + bytes_out + 256 + ws_bytes + 1024;
  if (cudaMalloc(reinterpret_cast<void**>(&d), total) != cudaSuccess) return fail("device allocation failed");
  std::size_t off = 0;
  const auto carve = [&](std::size_t n) {
    char* p = d + off;
    off += (n + 255) & ~std::size_t(255);
    return p;
  };
  double* d_m = reinterpret_cast<double*>(carve(bytes_m));
  float* d_lib = T > 0 ? reinterpret_cast<float*>(carve(bytes_lib)) : nullptr;
  float* d_out = reinterpret_cast<float*>(carve(bytes_out));
  int* d_status = reinterpret_cast<int*>(carve(sizeof(int)));
  void* d_ws = ws_bytes ? carve(ws_bytes) : nullptr;

  std::vector<float> host(n32);
  int status = 0;
  cudaError_t e = cudaMemcpy(d_m, m.data(), bytes_m, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && T > 0) e = cudaMemcpy(d_lib, lib.data(), bytes_lib, cudaMemcpyHostToDevice);
  int st = e == cudaSuccess ? hsi_build_statistics(1, B, T, diagonal_loading, d_m, d_lib, 0, nullptr, d_out,
                                                   nullptr, d_status, d_ws, ws_bytes, nullptr)
                            : static_cast<int>(e);
  if (st == HSI_OK) st = static_cast<int>(cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st == HSI_OK) st = static_cast<int>(cudaMemcpy(host.data(), d_out, bytes_out, cudaMemcpyDeviceToHost));
  cudaFree(d);
  if (st != HSI_OK) return fail(std::string("build_statistics: ") + hsi_status_string(st));
  switch (status) {
    case HSI_OK: break;
    case HSI_E_EMPTY: return fail("no scene statistics accumulated yet");
    case HSI_E_NOT_POSITIVE_DEFINITE:
      return fail("scene covariance is not positive definite at loading " + loading_text(diagonal_loading) +
                  "; neighbouring bands are nearly collinear, so raise the diagonal loading");
    case HSI_E_CORRELATION_NOT_PD:
      return fail("scene autocorrelation is not positive definite at loading " + loading_text(diagonal_loading) +
                  "; raise the diagonal loading");
    default: return fail(std::string("build_statistics: ") + hsi_status_string(status));
  }
  unpack(host.data(), B, T, out);
  out->valid = true;
  return true;
}

}  // namespace hsi
