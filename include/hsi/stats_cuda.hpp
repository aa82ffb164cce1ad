// hsi/stats_cuda.hpp - scene moments on the GPU.
//
// Drop-in for the reference's include/hsi/stats_cuda.hpp:26-72: FP64
// accumulators on the device that successive launch_accumulate_* calls add
// into, then read_moments to rebuild raw moments on the host.  Each
// accumulation runs the exact tensor-core moments pass (hsi_scene_moments)
// and adds its sums about `d_reference` (hsi_accumulate_shifted_moments).
#pragma once

#include <cuda_runtime.h>

#include "hsi/linalg.hpp"
#include "hsi/types.hpp"

namespace hsi {

inline std::size_t moment_outer_elements(int bands) {
  return static_cast<std::size_t>(bands) * static_cast<std::size_t>(bands);
}

// d_sum[bands] = 0, d_sum_outer[bands * bands] = 0.
cudaError_t launch_reset_moments(double* d_sum, double* d_sum_outer, int bands, cudaStream_t stream);

// d_sum += sum over pixels of x (BSQ fp32 cube at bsq_plane_stride).
cudaError_t launch_accumulate_mean(const float* d_cube_bsq, CubeShape shape, double* d_sum, cudaStream_t stream);

// d_sum += sum(x - r); lower triangle of d_sum_outer += sum (x - r)(x - r)^T.
// d_reference (bands floats, device) nullable: r = 0.
cudaError_t launch_accumulate_moments(const float* d_cube_bsq, CubeShape shape, const float* d_reference,
                                      double* d_sum, double* d_sum_outer, cudaStream_t stream);

// Synchronous: copy the accumulators back and rebuild raw moments about the
// host `reference` (nullable) with `count` pixels.
cudaError_t read_moments(const double* d_sum, const double* d_sum_outer, int bands, double count,
                         const float* reference, SpectralMoments* out);

// Full passes over the cube one accumulation makes (a strided subsample for
// the fixed-point range, then one streaming pass).
int moment_cube_reads(int bands);

}  // namespace hsi
