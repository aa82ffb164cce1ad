// hsi/sam_cuda.hpp - SAM scoring on the GPU.
//
// Drop-in for the reference's include/hsi/sam_cuda.hpp: the same functions
// with the same arguments, return codes and ownership (the caller owns every
// device buffer).  Implemented over the C ABI (include/hsi_b200.h): every
// variant runs the one B200 scoring kernel (hsi_score_frames).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "hsi/types.hpp"

namespace hsi {

// reference include/hsi/sam_cuda.hpp:18-36.  Baseline and Optimized score an
// fp32 BSQ cube, Half an fp16 BSQ cube, BipDirect an fp32 BIP cube (packed,
// in one pass: the transpose is fused into the scorer, hsi_sam_bip).
enum class SamVariant {
  Baseline,
  Optimized,
  Half,
  BipDirect,
};

const char* to_string(SamVariant variant);
bool parse_sam_variant(const std::string& name, SamVariant* out);

// Elements between band planes of a device cube: pixels rounded up to a
// multiple of 32 (the reference rounds to 8), so that every plane starts on
// a 128-byte boundary for the bulk-copy engine.
std::size_t bsq_plane_stride(CubeShape shape);

inline std::size_t bsq_device_elements(CubeShape shape) {
  return bsq_plane_stride(shape) * static_cast<std::size_t>(shape.bands);
}

// Largest num_targets * bands upload_targets accepts.  The library travels
// with each launch (no __constant__ state), so this only bounds the check.
int max_constant_target_elements();

// Validates a library for the launches that follow.  The reference copies it
// to __constant__ memory; here launch_sam_best reads d_targets and
// d_target_norms directly, so nothing is kept.  cudaErrorInvalidValue for an
// empty or oversized library.
cudaError_t upload_targets(const float* values, const float* norms, int num_targets, int bands);

// Best-matching target per pixel: d_score = smallest spectral angle (radians),
// d_target_id (nullable) = its index, lowest on ties; zero-norm pixels or
// targets score pi/2.  reference include/hsi/sam_cuda.hpp:91-96.
cudaError_t launch_sam_best(SamVariant variant, const void* d_cube, CubeShape shape, const float* d_targets,
                            const float* d_target_norms, int num_targets, float* d_score,
                            std::int32_t* d_target_id, cudaStream_t stream, int opt_pixels_per_thread = 0);

// Every target's angle map: d_maps + t * map_stride.  No counterpart in the
// reference GPU API (its per-target maps are CPU-only, sam_cpu).
cudaError_t launch_sam_maps(const void* d_cube, CubeShape shape, bool half, const float* d_targets,
                            const float* d_target_norms, int num_targets, float* d_maps, std::size_t map_stride,
                            cudaStream_t stream);

cudaError_t launch_transpose_bip_to_bsq(const float* d_src, float* d_dst, CubeShape shape, cudaStream_t stream);

cudaError_t launch_narrow_to_half(const float* d_src, void* d_dst, std::size_t count, cudaStream_t stream);

// Scratch of the launchers whose reference signatures take no workspace
// (launch_detect, the moment accumulators, launch_rx_ace).  No counterpart in the reference.  Each (device, stream)
// keeps one device buffer between calls, grown only when a call needs more
// than earlier calls on that stream did: steady-state calls allocate nothing,
// and a graph may capture them once one call at the largest size has run
// outside the capture.  This waits for the devices and frees every such
// buffer (call it when the streams are done, e.g. before exit or between
// workloads of very different sizes).
cudaError_t release_launch_workspaces();

}  // namespace hsi
