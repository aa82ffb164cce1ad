// hsi/detect_cuda.hpp - threshold + NMS + compaction on the GPU.
//
// Drop-in for the reference's include/hsi/detect_cuda.hpp:16-19.  Semantics
// are those of the reference CPU path (detect_cpu, src/sam_cpu.cpp:86-138):
// polarity honoured, list in raster order, identical run to run.  *d_count is
// zeroed by the caller and receives the number found, which may exceed
// params.max_detections (only that many are written).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "hsi/types.hpp"

namespace hsi {

// Scratch is the stream's grow-only launch workspace (release_launch_workspaces
// in hsi/sam_cuda.hpp): after the first call at the largest map size on a
// stream, calls allocate nothing.
cudaError_t launch_detect(const float* d_score, const std::int32_t* d_target_id, CubeShape shape,
                          DetectionParams params, Detection* d_out, unsigned int* d_count, cudaStream_t stream);

}  // namespace hsi
