// hsi/types.hpp - the value types of the hsi detection API.
//
// Drop-in for the reference's include/hsi/types.hpp: the same names, fields
// and meanings, because callers of the reference construct and read these
// directly (shape, library, detection list, detection parameters).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace hsi {

// Memory order of a cube (reference include/hsi/types.hpp:17-21).
enum class Interleave {
  Bsq,  // band[b][y][x]
  Bil,  // line[y][b][x]
  Bip,  // pixel[y][x][b]
};

const char* to_string(Interleave interleave);

// Cube dimensions (reference include/hsi/types.hpp:27-46).
struct CubeShape {
  int height = 0;
  int width = 0;
  int bands = 0;

  std::size_t pixels() const { return static_cast<std::size_t>(height) * static_cast<std::size_t>(width); }
  std::size_t elements() const { return pixels() * static_cast<std::size_t>(bands); }
  std::size_t bytes_f32() const { return elements() * sizeof(float); }
  bool valid() const { return height > 0 && width > 0 && bands > 0; }
  bool operator==(const CubeShape& o) const { return height == o.height && width == o.width && bands == o.bands; }
  bool operator!=(const CubeShape& o) const { return !(*this == o); }
};

// A host frame (reference include/hsi/types.hpp:54-68).
struct HsiFrame {
  CubeShape shape;
  Interleave interleave = Interleave::Bsq;
  std::vector<float> data;
  std::uint64_t index = 0;
  double timestamp_s = 0.0;
  std::vector<float> wavelengths_nm;

  std::size_t offset(int band, int y, int x) const;
  float at(int band, int y, int x) const { return data[offset(band, y, x)]; }
};

struct Spectrum {
  std::string name;
  std::vector<float> values;
  std::vector<float> wavelengths_nm;

  int bands() const { return static_cast<int>(values.size()); }
};

// Target library (reference include/hsi/types.hpp:85-99).
struct SpectralLibrary {
  std::vector<Spectrum> targets;

  int size() const { return static_cast<int>(targets.size()); }
  int bands() const { return targets.empty() ? 0 : targets.front().bands(); }
  // target-major num_targets x bands
  std::vector<float> flatten() const;
  // L2 norm of each target, accumulated in double
  std::vector<float> norms() const;
};

// One detection, 16 bytes (reference include/hsi/types.hpp:101-106); the
// same layout as hsi_detection of the C ABI.
struct Detection {
  int x = 0;
  int y = 0;
  int target = 0;
  float score = 0;
};

enum class ScorePolarity {
  LowerIsBetter,
  HigherIsBetter,
};

const char* to_string(ScorePolarity polarity);

// reference include/hsi/types.hpp:122-140
struct DetectionParams {
  float threshold = 0.10f;
  int nms_radius = 2;
  int max_detections = 4096;
  ScorePolarity polarity = ScorePolarity::LowerIsBetter;
};

// Host re-interleaving of a cube (`src` and `dst` must not alias), and of a
// frame in place.
void convert_interleave(const float* src, float* dst, CubeShape shape, Interleave from, Interleave to);
void convert_frame(HsiFrame& frame, Interleave to);

}  // namespace hsi
