// hsi/envi.hpp - ENVI cubes from disk.
//
// Drop-in for the reference's include/hsi/envi.hpp:11-47: the same header
// rules, sample types, full-scale rescale and errors, so that a cube reads
// to the same floats as with the reference.
//
// Header (`key = value` per line; a value that opens with '{' runs to the
// matching '}' across lines; keys are case-insensitive; a key that starts
// with ';' makes its line a comment):
//   required: samples (width), lines (height), bands, data type;
//   optional: header offset (bytes before the data), byte order (0 little,
//   else big), interleave (bsq, bil, bip), wavelength (a list; any entry that
//   is not a number empties it).
// Data types: 1 u8, 2 i16, 3 i32, 4 f32, 5 f64, 12 u16, 13 u32.  Integer
// samples become float and are multiplied by 1 / full scale (255, 32767,
// 65535, 2147483647 for both 32-bit types), so one threshold serves every bit
// depth; float samples pass through.
// The data file sits beside the header, named like the header without its
// ".hdr" with one of: no extension, .float .dat .img .bin .raw .bsq .bil
// .bip .cube (tried in that order).
#pragma once

#include <cstddef>
#include <map>
#include <string>
#include <vector>

#include "hsi/types.hpp"

namespace hsi {

struct EnviHeader {
  CubeShape shape;
  Interleave interleave = Interleave::Bsq;
  int data_type = 4;  // ENVI code, see above
  long header_offset = 0;
  bool little_endian = true;
  std::vector<float> wavelengths_nm;
  std::map<std::string, std::string> fields;  // every field, keys lower-case, values trimmed

  // Bytes per sample of data_type; throws std::runtime_error for a type not listed above.
  std::size_t sample_size() const;
};

// Throws std::runtime_error when the file cannot be read, a required field is
// missing or not an integer, a '{' is not closed, the interleave is unknown
// or the data type unsupported.
EnviHeader parse_envi_header(const std::string& hdr_path);

// The data file of `hdr_path`, or "" when none of the candidates exists.
std::string find_envi_data_file(const std::string& hdr_path);

// The cube as float32 in interleave `to`.  Throws std::runtime_error as
// parse_envi_header does, and when the data file is missing or shorter than
// header offset + height * width * bands samples.
HsiFrame read_envi(const std::string& hdr_path, Interleave to = Interleave::Bsq);

}  // namespace hsi
