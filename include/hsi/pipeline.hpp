// hsi/pipeline.hpp - the streaming SAM detection pipeline.
//
// Drop-in for the reference's include/hsi/pipeline.hpp:16-120: the same
// options, per-frame results and statistics.  Each of `num_streams` slots
// owns a pinned host cube, a device cube, score/target maps and a detection
// list; frame i runs in slot i % num_streams (upload, score, detect,
// download on the slot's stream) while the host fills the next slot, and
// results are delivered in frame order.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "hsi/frame_source.hpp"
#include "hsi/sam_cuda.hpp"
#include "hsi/types.hpp"

namespace hsi {

// Copy: frames are uploaded into HBM.  ZeroCopy (kernels reading mapped host
// memory) is rejected by Pipeline::create: the scoring kernel streams the
// cube with bulk copies from device memory.
enum class MemoryMode {
  Copy,
  ZeroCopy,
};

const char* to_string(MemoryMode mode);
bool parse_memory_mode(const std::string& name, MemoryMode* out);

struct PipelineOptions {
  SamVariant variant = SamVariant::Optimized;
  MemoryMode memory = MemoryMode::Copy;
  DetectionParams detection;
  int num_streams = 3;
  int prefill = 0;             // frames read from the source before timing starts
  bool time_stages = true;     // per-stage CUDA event timing
  bool return_score_map = false;
};

struct FrameResult {
  FrameMeta meta;
  std::vector<Detection> detections;
  unsigned int detections_found = 0;  // may exceed detections.size() if saturated
  std::vector<float> score_map;
  float ms_source = 0;
  float ms_upload = 0;
  float ms_score = 0;
  float ms_detect = 0;
  float ms_download = 0;
  float ms_gpu = 0;
  float ms_wall = 0;
};

struct PipelineStats {
  std::uint64_t frames = 0;
  double wall_s = 0;
  double fps = 0;
  double cube_gb_per_s = 0;
  double mpixel_per_s = 0;
  float ms_p50 = 0, ms_p95 = 0, ms_p99 = 0, ms_max = 0;
  float mean_source = 0, mean_upload = 0, mean_score = 0, mean_detect = 0, mean_download = 0, mean_gpu = 0;
  std::uint64_t total_detections = 0;
};

class Pipeline {
 public:
  virtual ~Pipeline() = default;
  // nullptr with *error set when the options, source or library are unusable
  // or a device allocation fails.
  static std::unique_ptr<Pipeline> create(FrameSource* source, const SpectralLibrary& library,
                                          const PipelineOptions& options, std::string* error);
  // Run `frames` frames (0: until the source ends); on_frame sees each result
  // in order.  false with *error on a CUDA failure.
  virtual bool run(std::uint64_t frames, const std::function<void(const FrameResult&)>& on_frame,
                   std::string* error) = 0;
  virtual PipelineStats stats() const = 0;
  virtual std::string describe() const = 0;
};

}  // namespace hsi
