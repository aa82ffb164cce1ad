"""The C-ABI library loads and exports every entry point include/*.h declares.

No compute calls: these run without a GPU."""
import ctypes as C
import glob
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "hsi-detectors-cuda_b200", "hsi_b200", "libhsi_b200.so")


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"HSI_API\s+[\w\s\*]+?\b(hsi_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "hsi_score_frames" in names and "hsi_detect" in names and len(names) >= 9


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.fail(f"{LIB} not built (run `make -C hsi-detectors-cuda_b200`)")
    lib = C.CDLL(LIB)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_host_only_entry_points_work_without_a_gpu():
    import hsi_b200
    assert hsi_b200.version() >= 100
    assert hsi_b200.plane_stride(520, 696) == 361920
    assert hsi_b200.plane_stride(3, 5) == 32
    assert hsi_b200.plane_stride(0, 5) == 0
    assert "positive definite" in hsi_b200.status_string(hsi_b200.E_NOT_POSITIVE_DEFINITE)
    sc = hsi_b200.scene(113, n_targets=8)
    spectra = hsi_b200.scene_spectra(sc)
    assert spectra.shape == (6 + 8 + 1, 113) and spectra.min() >= 0
    assert hsi_b200.detect_workspace_bytes(1024, 1024) > 0


def test_device_spectra_match_oracle_spectra():
    """Host-side spectra are double-precision and must agree exactly with the
    oracle's generator (both come from csrc/synth.h)."""
    import numpy as np
    import hsi_b200
    import oracle
    sc = hsi_b200.scene(64, n_targets=5, library_seed=1234)
    em, tg, an = oracle.scene_spectra(1234, 64, 6, 5)
    sp = hsi_b200.scene_spectra(sc)
    np.testing.assert_array_equal(sp[:6], em)
    np.testing.assert_array_equal(sp[6:11], tg)
    np.testing.assert_array_equal(sp[11], an)
