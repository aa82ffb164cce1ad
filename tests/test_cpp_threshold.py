"""CPU: the C++ layer's chi-squared RX threshold equals the reference's.

hsi::rx_threshold_for_false_alarm_rate (libhsi_cxx.so, the drop-in for
src/detectors_cpu.cpp:189-206) is compared bit for bit with the reference's own
function compiled from its sources (oracle/_ref), over band counts of every
configuration (16, 113, 224) and a few more, and rates from 0.5 down to 1e-9.
No GPU is used: the function is host code.
"""
import ctypes as C
import os

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CXXLIB = os.path.join(REPO, "hsi-detectors-cuda_b200", "hsi_b200", "libhsi_cxx.so")
MANGLED = "_ZN3hsi33rx_threshold_for_false_alarm_rateEid"  # hsi::rx_threshold_for_false_alarm_rate(int, double)


@pytest.fixture(scope="module")
def product_threshold():
    if not os.path.exists(CXXLIB):
        pytest.fail("libhsi_cxx.so is missing: build the package first")
    fn = getattr(C.CDLL(CXXLIB), MANGLED)
    fn.argtypes = [C.c_int, C.c_double]
    fn.restype = C.c_double
    return fn


@pytest.mark.parametrize("bands", [1, 2, 3, 16, 113, 127, 224, 256])
def test_rx_threshold_equals_reference(orc, product_threshold, bands):
    if not orc.ref_available():
        pytest.fail("oracle/_ref is missing: run oracle/Makefile")
    for rate in (0.5, 0.1, 1e-2, 1e-3, 1e-4, 1e-6, 1e-9):
        want = orc.ref_rx_threshold(bands, rate)
        got = product_threshold(bands, rate)
        assert got == want, f"B={bands} rate={rate}: {got!r} != {want!r}"
