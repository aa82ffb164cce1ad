// envi.cpp - ENVI header parsing and cube reading (include/hsi/envi.hpp).
// The rules follow the reference's src/envi.cpp:92-260 so that files read the
// same; the code is this library's.
#include "hsi/envi.hpp"

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <memory>
#include <stdexcept>

#include "hsi/frame_source.hpp"

namespace hsi {
namespace {

bool blank(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }

std::string trimmed(const std::string& s, std::size_t begin, std::size_t end) {
  while (begin < end && blank(s[begin])) ++begin;
  while (end > begin && blank(s[end - 1])) --end;
  return s.substr(begin, end - begin);
}

std::string lowered(std::string s) {
  for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return s;
}

// Entries of a brace list: separated by commas or line breaks, trimmed, empty ones dropped.
std::vector<std::string> list_entries(const std::string& body) {
  std::vector<std::string> out;
  std::size_t start = 0;
  for (std::size_t i = 0; i <= body.size(); ++i) {
    if (i == body.size() || body[i] == ',' || body[i] == '\n' || body[i] == '\r') {
      std::string t = trimmed(body, start, i);
      if (!t.empty()) out.push_back(std::move(t));
      start = i + 1;
    }
  }
  return out;
}

int required_int(const std::map<std::string, std::string>& f, const std::string& key) {
  const auto it = f.find(key);
  if (it == f.end()) throw std::runtime_error("ENVI header is missing required field '" + key + "'");
  try {
    return std::stoi(it->second);
  } catch (const std::exception&) {
    throw std::runtime_error("ENVI field '" + key + "' is not an integer: " + it->second);
  }
}

// Sample i of a raw buffer as float, byte-swapped when `swap`.
template <typename T>
float sample(const unsigned char* raw, std::size_t i, bool swap) {
  unsigned char b[sizeof(T)];
  std::memcpy(b, raw + i * sizeof(T), sizeof(T));
  if (swap)
    for (std::size_t k = 0; k < sizeof(T) / 2; ++k) {
      const unsigned char t = b[k];
      b[k] = b[sizeof(T) - 1 - k];
      b[sizeof(T) - 1 - k] = t;
    }
  T v;
  std::memcpy(&v, b, sizeof(T));
  return static_cast<float>(v);
}

template <typename T>
void decode_all(const unsigned char* raw, std::size_t n, bool swap, float scale, float* out) {
  for (std::size_t i = 0; i < n; ++i) out[i] = sample<T>(raw, i, swap) * scale;
}

bool little_endian_host() {
  const std::uint32_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

}  // namespace

std::size_t EnviHeader::sample_size() const {
  switch (data_type) {
    case 1: return 1;
    case 2: case 12: return 2;
    case 3: case 4: case 13: return 4;
    case 5: return 8;
    default: throw std::runtime_error("unsupported ENVI data type " + std::to_string(data_type));
  }
}

EnviHeader parse_envi_header(const std::string& hdr_path) {
  std::ifstream in(hdr_path);
  if (!in) throw std::runtime_error("cannot open ENVI header: " + hdr_path);
  const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  EnviHeader h;
  // Scan for '=' rather than by lines: a brace list (wavelengths) wraps.
  std::size_t pos = 0;
  while (pos < text.size()) {
    const std::size_t eq = text.find('=', pos);
    if (eq == std::string::npos) break;
    const std::size_t nl = text.rfind('\n', eq);
    const std::size_t key_begin = nl == std::string::npos ? 0 : nl + 1;
    const std::string key = lowered(trimmed(text, key_begin, eq));
    if (!key.empty() && key[0] == ';') {  // a comment line
      const std::size_t eol = text.find('\n', eq);
      pos = eol == std::string::npos ? text.size() : eol + 1;
      continue;
    }
    std::size_t v = eq + 1;
    while (v < text.size() && (text[v] == ' ' || text[v] == '\t')) ++v;
    if (v >= text.size()) break;
    std::string value;
    if (text[v] == '{') {
      const std::size_t close = text.find('}', v);
      if (close == std::string::npos) throw std::runtime_error("unterminated '{' in ENVI header: " + hdr_path);
      value = trimmed(text, v + 1, close);
      pos = close + 1;
    } else {
      const std::size_t eol = text.find('\n', v);
      const std::size_t stop = eol == std::string::npos ? text.size() : eol;
      value = trimmed(text, v, stop);
      pos = stop + 1;
    }
    if (!key.empty()) h.fields[key] = value;
  }
  h.shape.width = required_int(h.fields, "samples");
  h.shape.height = required_int(h.fields, "lines");
  h.shape.bands = required_int(h.fields, "bands");
  h.data_type = required_int(h.fields, "data type");
  auto it = h.fields.find("header offset");
  if (it != h.fields.end()) h.header_offset = std::stol(it->second);
  it = h.fields.find("byte order");
  if (it != h.fields.end()) h.little_endian = std::stoi(it->second) == 0;
  it = h.fields.find("interleave");
  if (it != h.fields.end()) {
    const std::string il = lowered(it->second);
    if (il == "bsq")
      h.interleave = Interleave::Bsq;
    else if (il == "bil")
      h.interleave = Interleave::Bil;
    else if (il == "bip")
      h.interleave = Interleave::Bip;
    else
      throw std::runtime_error("unknown ENVI interleave '" + il + "'");
  }
  it = h.fields.find("wavelength");
  if (it != h.fields.end()) {
    for (const std::string& e : list_entries(it->second)) {
      try {
        h.wavelengths_nm.push_back(std::stof(e));
      } catch (const std::exception&) {
        h.wavelengths_nm.clear();  // not a list of numbers after all
        break;
      }
    }
  }
  (void)h.sample_size();  // rejects an unsupported data type here
  return h;
}

std::string find_envi_data_file(const std::string& hdr_path) {
  std::string stem = hdr_path;
  if (stem.size() > 4 && lowered(stem.substr(stem.size() - 4)) == ".hdr") stem.resize(stem.size() - 4);
  for (const char* ext : {"", ".float", ".dat", ".img", ".bin", ".raw", ".bsq", ".bil", ".bip", ".cube"}) {
    const std::string candidate = stem + ext;
    if (std::ifstream(candidate, std::ios::binary)) return candidate;
  }
  return "";
}

HsiFrame read_envi(const std::string& hdr_path, Interleave to) {
  const EnviHeader h = parse_envi_header(hdr_path);
  const std::string data_path = find_envi_data_file(hdr_path);
  if (data_path.empty()) throw std::runtime_error("no ENVI data file found alongside " + hdr_path);
  const std::size_t size = h.sample_size();
  const std::size_t n = h.shape.elements();
  const std::size_t need = n * size;
  std::ifstream in(data_path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot open ENVI data file: " + data_path);
  in.seekg(0, std::ios::end);
  const std::size_t file_bytes = static_cast<std::size_t>(in.tellg());
  if (file_bytes < need + static_cast<std::size_t>(h.header_offset))
    throw std::runtime_error("ENVI data file " + data_path + " is " + std::to_string(file_bytes) + " bytes, need " +
                             std::to_string(need + h.header_offset));
  in.seekg(h.header_offset, std::ios::beg);
  std::vector<unsigned char> raw(need);
  in.read(reinterpret_cast<char*>(raw.data()), static_cast<std::streamsize>(need));
  if (!in) throw std::runtime_error("short read on ENVI data file: " + data_path);
  const bool swap = h.little_endian != little_endian_host();
  HsiFrame frame;
  frame.shape = h.shape;
  frame.interleave = h.interleave;
  frame.wavelengths_nm = h.wavelengths_nm;
  frame.data.resize(n);
  float* out = frame.data.data();
  switch (h.data_type) {
    case 1: decode_all<std::uint8_t>(raw.data(), n, false, 1.0f / 255.0f, out); break;
    case 2: decode_all<std::int16_t>(raw.data(), n, swap, 1.0f / 32767.0f, out); break;
    case 12: decode_all<std::uint16_t>(raw.data(), n, swap, 1.0f / 65535.0f, out); break;
    case 3: decode_all<std::int32_t>(raw.data(), n, swap, 1.0f / 2147483647.0f, out); break;
    case 13: decode_all<std::uint32_t>(raw.data(), n, swap, 1.0f / 2147483647.0f, out); break;
    case 4: decode_all<float>(raw.data(), n, swap, 1.0f, out); break;
    default: decode_all<double>(raw.data(), n, swap, 1.0f, out); break;  // 5, the last the header admits
  }
  convert_frame(frame, to);
  return frame;
}

namespace {

// Resident BSQ cubes, copied out one per read at the caller's plane stride.
class EnviReplay final : public FrameSource {
 public:
  explicit EnviReplay(const EnviReplayOptions& o) : loop_(o.loop) {
    if (o.hdr_paths.empty()) throw std::invalid_argument("EnviReplaySource: no headers given");
    const std::size_t keep = static_cast<std::size_t>(std::max(1, o.max_resident));
    for (std::size_t i = 0; i < o.hdr_paths.size() && cubes_.size() < keep; ++i) {
      HsiFrame f = read_envi(o.hdr_paths[i], Interleave::Bsq);
      if (cubes_.empty()) {
        shape_ = f.shape;
      } else if (f.shape != shape_) {
        throw std::runtime_error("EnviReplaySource: " + o.hdr_paths[i] + " is " + std::to_string(f.shape.height) +
                                 "x" + std::to_string(f.shape.width) + "x" + std::to_string(f.shape.bands) +
                                 ", expected the shape of the first cube");
      }
      cubes_.push_back(std::move(f.data));
    }
  }

  CubeShape shape() const override { return shape_; }
  Interleave interleave() const override { return Interleave::Bsq; }
  std::uint64_t length() const override { return loop_ ? 0 : cubes_.size(); }

  bool read_into(float* dst, std::size_t plane_stride, FrameMeta* meta) override {
    if (next_ >= cubes_.size()) {
      if (!loop_) return false;
      next_ = 0;
    }
    const float* src = cubes_[next_].data();
    const std::size_t P = shape_.pixels();
    for (int b = 0; b < shape_.bands; ++b)
      std::memcpy(dst + static_cast<std::size_t>(b) * plane_stride, src + static_cast<std::size_t>(b) * P,
                  P * sizeof(float));
    if (meta) {
      meta->index = emitted_;
      meta->timestamp_s = static_cast<double>(emitted_) / 30.0;
    }
    ++next_;
    ++emitted_;
    return true;
  }

  void reset() override {
    next_ = 0;
    emitted_ = 0;
  }

  std::string describe() const override {
    return "envi-replay(" + std::to_string(cubes_.size()) + " cubes, " + std::to_string(shape_.height) + "x" +
           std::to_string(shape_.width) + "x" + std::to_string(shape_.bands) + ")";
  }

 private:
  bool loop_;
  CubeShape shape_;
  std::vector<std::vector<float>> cubes_;
  std::size_t next_ = 0;
  std::uint64_t emitted_ = 0;
};

}  // namespace

std::unique_ptr<FrameSource> make_envi_replay_source(const EnviReplayOptions& options) {
  return std::make_unique<EnviReplay>(options);
}

}  // namespace hsi
