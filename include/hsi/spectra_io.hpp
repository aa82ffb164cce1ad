// hsi/spectra_io.hpp - target libraries as plain CSV text.
//
// Drop-in for the reference's include/hsi/spectra_io.hpp:9-22, with the same
// file format and entry points:
//
//     # comment lines and blank lines are skipped
//     wavelength,400.0,410.0,420.0      (optional; "wavelengths" also accepted)
//     blood,0.11,0.19,0.24              (one row per target: name, then values)
//
// read_spectra_csv throws std::runtime_error, naming the file (and the line
// where there is one), when:
//   * the file cannot be opened;
//   * a row has no value after its name, or a value does not start with a
//     number (std::stof semantics, as the reference);
//   * no target row is found;
//   * the targets' band counts differ;
//   * the wavelength row's length differs from the band count.
// The wavelength row, when present, is copied to every target.
// write_spectra_csv writes floats with 9 significant digits, so a library
// reads back bit for bit.
#pragma once

#include <string>

#include "hsi/types.hpp"

namespace hsi {

SpectralLibrary read_spectra_csv(const std::string& path);

void write_spectra_csv(const std::string& path, const SpectralLibrary& library);

}  // namespace hsi
