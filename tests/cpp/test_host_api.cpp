// Host-only properties of the drop-in API (no device calls, so it runs on a
// machine without a GPU):
//   * the name parsers accept the reference's names and aliases
//     (src/sam.cu:320-336, src/pipeline.cu:444-456, src/detector.cpp:21-45);
//   * read_spectra_csv / write_spectra_csv follow the reference's CSV format
//     and error cases (src/spectra_io.cpp:27-122), and a written library reads
//     back bit for bit;
//   * make_envi_replay_source replays ENVI cubes as the reference's
//     EnviReplaySource does (src/frame_source.cpp:69-145).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "check.hpp"
#include "hsi/detector.hpp"
#include "hsi/envi.hpp"
#include "hsi/frame_source.hpp"
#include "hsi/pipeline.hpp"
#include "hsi/sam_cuda.hpp"
#include "hsi/spectra_io.hpp"

using namespace hsi;

namespace {

std::string temp_path(const char* name) { return std::string("/tmp/hsi_host_api_") + name; }

std::string write_file(const char* name, const std::string& text) {
  const std::string path = temp_path(name);
  std::ofstream(path) << text;
  return path;
}

// The message of the runtime_error that read_spectra_csv(path) throws, or "" if none.
std::string read_error(const std::string& path) {
  try {
    read_spectra_csv(path);
  } catch (const std::runtime_error& e) {
    return e.what();
  }
  return "";
}

bool contains(const std::string& s, const std::string& part) { return s.find(part) != std::string::npos; }

void test_variant_names() {
  SamVariant v = SamVariant::Baseline;
  CHECK(parse_sam_variant("optimized", &v) && v == SamVariant::Optimized);
  CHECK(parse_sam_variant("opt", &v) && v == SamVariant::Optimized);
  CHECK(parse_sam_variant("baseline", &v) && v == SamVariant::Baseline);
  CHECK(parse_sam_variant("half", &v) && v == SamVariant::Half);
  CHECK(parse_sam_variant("fp16", &v) && v == SamVariant::Half);
  CHECK(parse_sam_variant("bip", &v) && v == SamVariant::BipDirect);
  CHECK(!parse_sam_variant("Optimized", &v));
  CHECK(!parse_sam_variant("", &v));
  for (SamVariant x : {SamVariant::Baseline, SamVariant::Optimized, SamVariant::Half, SamVariant::BipDirect}) {
    SamVariant back = SamVariant::Baseline;
    CHECK(parse_sam_variant(to_string(x), &back) && back == x);
  }
  CHECK(std::string(to_string(SamVariant::Optimized)) == "optimized");
}

void test_memory_mode_names() {
  MemoryMode m = MemoryMode::Copy;
  CHECK(parse_memory_mode("zerocopy", &m) && m == MemoryMode::ZeroCopy);
  CHECK(parse_memory_mode("zero-copy", &m) && m == MemoryMode::ZeroCopy);
  CHECK(parse_memory_mode("copy", &m) && m == MemoryMode::Copy);
  CHECK(!parse_memory_mode("pinned", &m));
  CHECK(std::string(to_string(MemoryMode::ZeroCopy)) == "zerocopy");
}

void test_detector_names() {
  const char* names[] = {"sam", "rx", "ace", "cem"};
  const Detector kinds[] = {Detector::Sam, Detector::Rx, Detector::Ace, Detector::Cem};
  for (int i = 0; i < 4; ++i) {
    Detector d = Detector::Sam;
    CHECK(parse_detector(names[i], &d) && d == kinds[i]);
  }
  Detector d = Detector::Sam;
  CHECK(!parse_detector("SAM", &d));
}

void test_library_reads_the_reference_format() {
  const std::string path = write_file("lib.csv",
                                      "# field library\n"
                                      "\n"
                                      "wavelength, 400.0, 410.0, 420.0\n"
                                      "blood,0.11,0.19,0.24\r\n"
                                      "  tomato , 0.31,0.28,0.22,\n");
  const SpectralLibrary lib = read_spectra_csv(path);
  CHECK(lib.size() == 2);
  CHECK(lib.bands() == 3);
  CHECK(lib.targets[0].name == "blood");
  CHECK(lib.targets[1].name == "tomato");
  CHECK(lib.targets[0].values[1] == 0.19f);
  CHECK(lib.targets[1].values[2] == 0.22f);
  for (const Spectrum& s : lib.targets) CHECK(s.wavelengths_nm == std::vector<float>({400.0f, 410.0f, 420.0f}));
}

void test_library_errors_name_the_file_and_line() {
  CHECK(contains(read_error(temp_path("does_not_exist.csv")), "cannot open spectral library"));
  std::string e = read_error(write_file("short.csv", "a,1,2\nlonely\n"));
  CHECK(contains(e, "short.csv:2:") && contains(e, "expected a name followed by at least one value"));
  e = read_error(write_file("nan.csv", "a,1,x2\n"));
  CHECK(contains(e, "nan.csv:1:") && contains(e, "'x2' is not a number"));
  e = read_error(write_file("gap.csv", "a,1,,2\n"));
  CHECK(contains(e, "gap.csv:1:") && contains(e, "is not a number"));
  e = read_error(write_file("empty.csv", "# nothing\nwavelength,1,2\n"));
  CHECK(contains(e, "no target spectra found"));
  e = read_error(write_file("ragged.csv", "a,1,2,3\nb,1,2\n"));
  CHECK(contains(e, "target 'b' has 2 bands, expected 3"));
  e = read_error(write_file("wl.csv", "wavelength,1,2\na,1,2,3\n"));
  CHECK(contains(e, "wavelength row has 2 entries but the spectra have 3 bands"));
}

void test_library_round_trips_bit_for_bit() {
  SpectralLibrary lib;
  for (int t = 0; t < 3; ++t) {
    Spectrum s;
    s.name = "target" + std::to_string(t);
    for (int b = 0; b < 17; ++b) {
      s.values.push_back(1.0f / static_cast<float>(3 + 7 * t + b) + 1e-7f * static_cast<float>(b));
      s.wavelengths_nm.push_back(400.0f + 10.123f * static_cast<float>(b));
    }
    lib.targets.push_back(s);
  }
  const std::string path = temp_path("round.csv");
  write_spectra_csv(path, lib);
  const SpectralLibrary back = read_spectra_csv(path);
  CHECK(back.size() == lib.size());
  for (int t = 0; t < lib.size() && t < back.size(); ++t) {
    CHECK(back.targets[t].name == lib.targets[t].name);
    CHECK(back.targets[t].values == lib.targets[t].values);
    CHECK(back.targets[t].wavelengths_nm == lib.targets[t].wavelengths_nm);
  }
}

// A height x width x bands f32 BIP cube whose value at (b, y, x) is
// base + b * 1000 + y * 10 + x, written as <name>.hdr and <name>.
std::string write_bip_cube(const char* name, int h, int w, int bands, float base) {
  const std::string hdr = temp_path(name) + ".hdr";
  std::ofstream(hdr) << "ENVI\nsamples = " << w << "\nlines = " << h << "\nbands = " << bands
                     << "\ndata type = 4\ninterleave = bip\nbyte order = 0\n";
  std::vector<float> v;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x)
      for (int b = 0; b < bands; ++b) v.push_back(base + b * 1000.0f + y * 10.0f + x);
  std::ofstream(temp_path(name), std::ios::binary)
      .write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(float)));
  return hdr;
}

void test_envi_replay_cycles_resident_cubes() {
  const std::string a = write_bip_cube("replay_a", 3, 4, 2, 0.0f);
  const std::string b = write_bip_cube("replay_b", 3, 4, 2, 0.5f);
  const std::string c = write_bip_cube("replay_c", 3, 4, 2, 0.25f);
  EnviReplayOptions o;
  o.hdr_paths = {a, b, c};
  o.max_resident = 2;  // the third cube is never read
  o.loop = false;
  std::unique_ptr<FrameSource> src = make_envi_replay_source(o);
  CHECK(src->shape() == CubeShape({3, 4, 2}));
  CHECK(src->interleave() == Interleave::Bsq);
  CHECK(src->length() == 2);
  CHECK(src->describe() == "envi-replay(2 cubes, 3x4x2)");
  const std::size_t stride = 16;  // wider than the 12 pixels: planes land 16 floats apart
  std::vector<float> dst(stride * 2, -1.0f);
  FrameMeta meta;
  for (int f = 0; f < 2; ++f) {
    CHECK(src->read_into(dst.data(), stride, &meta));
    CHECK(meta.index == static_cast<std::uint64_t>(f));
    CHECK(meta.timestamp_s == f / 30.0);
    const float base = f == 0 ? 0.0f : 0.5f;
    for (int band = 0; band < 2; ++band)
      for (int y = 0; y < 3; ++y)
        for (int x = 0; x < 4; ++x) CHECK(dst[band * stride + y * 4 + x] == base + band * 1000.0f + y * 10.0f + x);
    CHECK(dst[12] == -1.0f);  // the stride padding is left alone
  }
  CHECK(!src->read_into(dst.data(), stride, &meta));
  src->reset();
  CHECK(src->read_into(dst.data(), stride, &meta) && meta.index == 0 && dst[0] == 0.0f);
  o.loop = true;
  o.max_resident = 1;
  std::unique_ptr<FrameSource> looped = make_envi_replay_source(o);
  CHECK(looped->length() == 0);
  for (int f = 0; f < 3; ++f) CHECK(looped->read_into(dst.data(), 12, &meta) && meta.index == static_cast<std::uint64_t>(f));
}

void test_envi_replay_rejects_what_the_reference_rejects() {
  bool threw = false;
  try {
    make_envi_replay_source(EnviReplayOptions{});
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  CHECK(threw);
  EnviReplayOptions o;
  o.hdr_paths = {write_bip_cube("shape_a", 3, 4, 2, 0.0f), write_bip_cube("shape_b", 3, 5, 2, 0.0f)};
  std::string message;
  try {
    make_envi_replay_source(o);
  } catch (const std::runtime_error& e) {
    message = e.what();
  }
  CHECK(contains(message, "is 3x5x2, expected the shape of the first cube"));
}

}  // namespace

int main() {
  test_variant_names();
  test_memory_mode_names();
  test_detector_names();
  test_library_reads_the_reference_format();
  test_library_errors_name_the_file_and_line();
  test_library_round_trips_bit_for_bit();
  test_envi_replay_cycles_resident_cubes();
  test_envi_replay_rejects_what_the_reference_rejects();
  return tcheck::finish("host_api");
}
