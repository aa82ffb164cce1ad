// hsi/frame_source.hpp - where frames come from.
//
// Drop-in for the reference's FrameSource interface
// (include/hsi/frame_source.hpp:19-57): the pipeline pulls frames through it
// into caller memory at a given plane stride.  The synthetic source here
// draws scenes from the library's own scene model (Dirichlet-mixed Gaussian-
// bump endmembers, implanted targets, anomalies, Gaussian noise; the model
// hsi_generate uses on the device), so a frame's pixels are the same wherever
// it is generated.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "hsi/types.hpp"

namespace hsi {

struct FrameMeta {
  std::uint64_t index = 0;
  double timestamp_s = 0.0;
};

class FrameSource {
 public:
  virtual ~FrameSource() = default;
  virtual CubeShape shape() const = 0;
  virtual Interleave interleave() const = 0;
  // Frames available; 0 means unbounded.
  virtual std::uint64_t length() const = 0;
  // Write the next frame as BSQ planes `plane_stride` floats apart; false at
  // the end of the stream.
  virtual bool read_into(float* dst, std::size_t plane_stride, FrameMeta* meta) = 0;
  virtual void reset() = 0;
  virtual std::string describe() const = 0;
  // Per-pixel truth of the last frame read (0 background, 1 + t target t,
  // 255 anomaly), when the source knows it.
  virtual const std::uint8_t* truth_mask() const { return nullptr; }
  // The implanted target library, when the source knows it.
  virtual const SpectralLibrary* library() const { return nullptr; }
};

// The synthetic scene source.  Field names follow the reference's
// SyntheticOptions (include/hsi/frame_source.hpp:72-82) where they mean the
// same thing; the scene model is this library's.
struct SyntheticOptions {
  CubeShape shape{512, 512, 128};
  int background_endmembers = 6;
  int num_targets = 3;
  float target_fraction = 0.005f;   // per-target implant probability per pixel
  float anomaly_fraction = 0.0f;
  float noise_sigma = 0.005f;
  std::uint64_t seed = 0x5EED0000;  // library seed; frame f uses seed + 1 + f
  std::uint64_t length = 0;         // 0 == unbounded
};
std::unique_ptr<FrameSource> make_synthetic_source(const SyntheticOptions& options);

// ENVI cubes replayed from disk (reference include/hsi/frame_source.hpp:60-69):
// the first max(1, max_resident) headers are read (read_envi, as BSQ) when the
// source is made, all of the first cube's shape, and frames cycle through them
// (or end after the last when !loop).  Frame i has index i and timestamp i / 30 s.
// Throws std::invalid_argument with no headers, std::runtime_error when a cube
// cannot be read or its shape differs from the first.
struct EnviReplayOptions {
  std::vector<std::string> hdr_paths;
  int max_resident = 4;
  bool loop = true;
};
std::unique_ptr<FrameSource> make_envi_replay_source(const EnviReplayOptions& options);

}  // namespace hsi
