// envi_dump <header> <to: 0 BSQ, 1 BIL, 2 BIP> <out>: hsi::read_envi of the
// header, written to <out> as int32 {height, width, bands, wavelength count},
// the cube's floats, then the wavelengths.  A read error prints
// "error: <message>" to stderr and exits 3.  Host only (no device calls).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>

#include "hsi/envi.hpp"

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: envi_dump <header> <to> <out>\n");
    return 2;
  }
  try {
    const hsi::HsiFrame f = hsi::read_envi(argv[1], static_cast<hsi::Interleave>(std::atoi(argv[2])));
    std::FILE* out = std::fopen(argv[3], "wb");
    if (!out) return 4;
    const std::int32_t dims[4] = {f.shape.height, f.shape.width, f.shape.bands,
                                  static_cast<std::int32_t>(f.wavelengths_nm.size())};
    bool ok = std::fwrite(dims, sizeof(dims), 1, out) == 1;
    if (!f.data.empty()) ok = ok && std::fwrite(f.data.data(), sizeof(float), f.data.size(), out) == f.data.size();
    if (!f.wavelengths_nm.empty())
      ok = ok && std::fwrite(f.wavelengths_nm.data(), sizeof(float), f.wavelengths_nm.size(), out) ==
                     f.wavelengths_nm.size();
    ok = (std::fclose(out) == 0) && ok;
    return ok ? 0 : 4;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
}
