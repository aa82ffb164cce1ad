"""The C++ drop-in API (include/hsi/*.hpp, libhsi_cxx.so over the C ABI).

CPU: the library and the C++ test programs (tests/cpp) build, and the library
exports the reference's entry points under their reference names.
GPU: each test program runs the reference's SAM / detection / statistics /
pipeline properties through that API on the device and exits 0.
"""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "hsi-detectors-cuda_b200")
CXXLIB = os.path.join(PKG, "hsi_b200", "libhsi_cxx.so")
BIN = os.path.join(PKG, "build", "tests")
PROGRAMS = ["test_sam_gpu", "test_detector_gpu", "test_pipeline_gpu"]

# the reference's hsi:: entry points (include/hsi/*.hpp) the drop-in provides
REFERENCE_NAMES = [
    "hsi::launch_sam_best(", "hsi::upload_targets(", "hsi::bsq_plane_stride(",
    "hsi::max_constant_target_elements(", "hsi::launch_transpose_bip_to_bsq(", "hsi::launch_narrow_to_half(",
    "hsi::parse_sam_variant(", "hsi::launch_detect(", "hsi::launch_reset_moments(",
    "hsi::launch_accumulate_mean(", "hsi::launch_accumulate_moments(", "hsi::read_moments(",
    "hsi::moment_cube_reads(", "hsi::build_statistics(", "hsi::traits_of(", "hsi::parse_detector(",
    "hsi::rx_threshold_for_false_alarm_rate(", "hsi::Pipeline::create(", "hsi::make_synthetic_source(",
    "hsi::moments_from_shifted(", "hsi::SpectralLibrary::flatten(", "hsi::SpectralLibrary::norms(",
    "hsi::convert_interleave(", "hsi::parse_memory_mode(", "hsi::read_spectra_csv(", "hsi::write_spectra_csv(",
    "hsi::read_envi(", "hsi::parse_envi_header(", "hsi::find_envi_data_file(", "hsi::make_envi_replay_source(",
]


def _make_tests():
    subprocess.run(["make", "-s", "-j8", "-C", PKG, "all", "tests"], check=True, capture_output=True, text=True)


def test_cpp_library_and_tests_build():
    _make_tests()
    assert os.path.exists(CXXLIB)
    for p in PROGRAMS:
        assert os.access(os.path.join(BIN, p), os.X_OK), p


def test_cpp_library_exports_the_reference_entry_points():
    _make_tests()
    out = subprocess.run(["nm", "-DC", "--defined-only", CXXLIB], check=True, capture_output=True, text=True).stdout
    missing = [n for n in REFERENCE_NAMES if n not in out]
    assert not missing, missing


def test_host_only_program_passes_without_a_device():
    """Name parsers and the CSV library reader: no device calls."""
    _make_tests()
    r = subprocess.run([os.path.join(BIN, "test_host_api")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().splitlines()[-1] == "ok host_api", r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("program", PROGRAMS)
def test_cpp_program_passes_on_the_device(program):
    _make_tests()
    r = subprocess.run([os.path.join(BIN, program)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().splitlines()[-1].startswith("ok "), r.stdout
