// spectra_io.cpp - the CSV target library reader and writer
// (include/hsi/spectra_io.hpp; format of the reference's src/spectra_io.cpp:27-122).
#include "hsi/spectra_io.hpp"

#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace hsi {
namespace {

// [begin, end) of `s` without leading and trailing blanks.
std::string strip(const std::string& s, std::size_t begin, std::size_t end) {
  while (begin < end && (s[begin] == ' ' || s[begin] == '\t' || s[begin] == '\r' || s[begin] == '\n')) ++begin;
  while (end > begin && (s[end - 1] == ' ' || s[end - 1] == '\t' || s[end - 1] == '\r' || s[end - 1] == '\n')) --end;
  return s.substr(begin, end - begin);
}

// Comma-separated fields of a line, each stripped.
std::vector<std::string> fields_of(const std::string& line) {
  std::vector<std::string> out;
  std::size_t start = 0;
  for (;;) {
    const std::size_t comma = line.find(',', start);
    if (comma == std::string::npos) {
      out.push_back(strip(line, start, line.size()));
      return out;
    }
    out.push_back(strip(line, start, comma));
    start = comma + 1;
  }
}

std::runtime_error line_error(const std::string& path, int line, const std::string& what) {
  return std::runtime_error(path + ":" + std::to_string(line) + ": " + what);
}

}  // namespace

SpectralLibrary read_spectra_csv(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open spectral library: " + path);
  SpectralLibrary library;
  std::vector<float> wavelengths;
  std::string line;
  for (int number = 1; std::getline(in, line); ++number) {
    const std::string row = strip(line, 0, line.size());
    if (row.empty() || row[0] == '#') continue;
    std::vector<std::string> f = fields_of(row);
    // a trailing comma leaves an empty last field, which is not a value
    if (f.size() > 1 && f.back().empty()) f.pop_back();
    if (f.size() < 2) throw line_error(path, number, "expected a name followed by at least one value");
    std::vector<float> values;
    values.reserve(f.size() - 1);
    for (std::size_t i = 1; i < f.size(); ++i) {
      // std::stof semantics, as the reference: a leading number is taken,
      // a field that does not start with one is an error
      float v = 0.0f;
      try {
        v = std::stof(f[i]);
      } catch (const std::exception&) {
        throw line_error(path, number, "'" + f[i] + "' is not a number");
      }
      values.push_back(v);
    }
    if (f[0] == "wavelength" || f[0] == "wavelengths") {
      wavelengths = std::move(values);
      continue;
    }
    Spectrum s;
    s.name = f[0];
    s.values = std::move(values);
    library.targets.push_back(std::move(s));
  }
  if (library.targets.empty()) throw std::runtime_error(path + ": no target spectra found");
  const int bands = library.bands();
  for (const Spectrum& s : library.targets) {
    if (s.bands() != bands)
      throw std::runtime_error(path + ": target '" + s.name + "' has " + std::to_string(s.bands()) +
                               " bands, expected " + std::to_string(bands));
  }
  if (!wavelengths.empty()) {
    if (static_cast<int>(wavelengths.size()) != bands)
      throw std::runtime_error(path + ": wavelength row has " + std::to_string(wavelengths.size()) +
                               " entries but the spectra have " + std::to_string(bands) + " bands");
    for (Spectrum& s : library.targets) s.wavelengths_nm = wavelengths;
  }
  return library;
}

void write_spectra_csv(const std::string& path, const SpectralLibrary& library) {
  std::FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw std::runtime_error("cannot write spectral library: " + path);
  bool ok = std::fputs("# hyperspectral target spectra\n", f) >= 0;
  auto row = [&](const std::string& name, const std::vector<float>& values) {
    ok = ok && std::fputs(name.c_str(), f) >= 0;
    for (float v : values) ok = ok && std::fprintf(f, ",%.9g", static_cast<double>(v)) > 0;
    ok = ok && std::fputc('\n', f) != EOF;
  };
  if (!library.targets.empty() && !library.targets.front().wavelengths_nm.empty())
    row("wavelength", library.targets.front().wavelengths_nm);
  for (const Spectrum& s : library.targets) row(s.name, s.values);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) throw std::runtime_error("cannot write spectral library: " + path);
}

}  // namespace hsi
