// hsi/detectors.hpp - RX, ACE and CEM scoring on the GPU.
//
// The reference scores RX, ACE and CEM on the CPU only (rx_cpu, ace_best_cpu,
// cem_best_cpu in include/hsi/detectors.hpp:22-56, src/detectors_cpu.cpp:
// 95-187).  These launchers compute the same maps, with the same rules, on
// the device from a frame's statistics:
//   RX      |W (x - mean)|^2
//   ACE_t   (z . u_t)^2 / (|u_t|^2 |z|^2), z = W (x - mean); a target with
//           |u_t|^2 <= 0, or a pixel with |z|^2 <= 0, scores 0; best = the
//           largest, lowest t on ties, clamped to [0, 1]; -1 if none is valid
//   CEM_t   w_t . x (uncentred); best = the largest, lowest t on ties
// Device statistics come from DeviceStatistics (FP64, built on the GPU from
// the frame's own moments).  All launches are asynchronous on `stream`.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "hsi/detector.hpp"
#include "hsi/types.hpp"

namespace hsi {

// A frame's statistics resident on the device: the packed FP64 layout of
// hsi_build_statistics plus the CEM filters.  Owns its device memory.
class DeviceStatistics {
 public:
  DeviceStatistics() = default;
  ~DeviceStatistics();
  DeviceStatistics(const DeviceStatistics&) = delete;
  DeviceStatistics& operator=(const DeviceStatistics&) = delete;

  // Moments of the BSQ cube (fp32 or fp16 at bsq_plane_stride) on the GPU,
  // then the FP64 factorisation against `library` at `diagonal_loading`.
  // Returns cudaSuccess, a CUDA error, or cudaErrorInvalidValue with *status
  // (nullable) set to the library's HSI_E_* code when the factorisation
  // failed (not positive definite, empty).  Synchronous.
  cudaError_t build(const void* d_cube, CubeShape shape, bool half, const SpectralLibrary& library,
                    double diagonal_loading, cudaStream_t stream, int* status = nullptr);

  int bands() const { return bands_; }
  int num_targets() const { return targets_; }
  const double* packed() const { return packed_; }       // FP64, hsi_statistics_elements
  const float* cem_weights() const { return cem_; }      // num_targets x bands
  // The float statistics, as the reference's build_statistics returns them.
  bool download(DetectorStatistics* out) const;

 private:
  void release();
  int bands_ = 0, targets_ = 0;
  double* packed_ = nullptr;
  double* moments_ = nullptr;
  float* cem_ = nullptr;
  float* library_ = nullptr;
  void* workspace_ = nullptr;
  std::size_t workspace_bytes_ = 0;
};

// RX map and, when num_targets > 0, the best ACE score / target and the
// per-target ACE maps; each output nullable.  Plain FP32 CUDA-core path.
cudaError_t launch_rx_ace(const void* d_cube, CubeShape shape, bool half, const DeviceStatistics& stats,
                          float* d_rx, float* d_ace_best, std::int32_t* d_ace_target, float* d_ace_maps,
                          std::size_t map_stride, cudaStream_t stream);

// CEM best response / target and per-target maps (each nullable).
cudaError_t launch_cem(const void* d_cube, CubeShape shape, bool half, const DeviceStatistics& stats,
                       float* d_best, std::int32_t* d_target, float* d_maps, std::size_t map_stride,
                       cudaStream_t stream);

// Chi-square quantile: the RX threshold whose false-alarm rate under the
// Gaussian background model is `rate` (reference src/detectors_cpu.cpp:
// 189-206).  Host scalar arithmetic.
double rx_threshold_for_false_alarm_rate(int bands, double rate);

}  // namespace hsi
