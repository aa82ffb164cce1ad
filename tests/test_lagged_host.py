"""CPU: the lagged-statistics runner rejects bad options before touching a
device (include/hsi_lagged.h): NULL with HSI_E_INVALID, for each kind of bad
option.  No GPU is needed: the checks run on the host first."""
import ctypes as C

import numpy as np
import pytest


def _create(hsi, **kw):
    tg = np.ones((4, 113), np.float32)
    base = dict(height=64, width=64, bands=113, dtype=hsi.F32, targets=tg.ctypes.data, num_targets=4,
                detectors=hsi.LAGGED_SAM_CEM | hsi.LAGGED_RX_ACE, loading=1e-6, sam_threshold=0.1,
                cem_threshold=0.5, ace_threshold=0.5, rx_false_alarm_rate=1e-3, nms_radius=2, capacity=16)
    base.update(kw)
    opt = hsi.LaggedOptions(**base)
    st = C.c_int(12345)
    h = hsi.cxx_lib().hsi_lagged_create(C.byref(opt), C.byref(st))
    return h, st.value, tg


@pytest.mark.parametrize("bad", [
    dict(height=0), dict(width=-1), dict(bands=0), dict(bands=257), dict(dtype=7), dict(targets=None),
    dict(num_targets=0), dict(num_targets=17), dict(detectors=0), dict(detectors=4), dict(loading=-1.0),
    dict(capacity=-1), dict(nms_radius=-1), dict(rx_false_alarm_rate=0.0), dict(rx_false_alarm_rate=1.0),
])
def test_lagged_create_rejects_bad_options(bad):
    import hsi_b200 as hsi
    h, st, _ = _create(hsi, **bad)
    assert h is None and st == hsi.E_INVALID


def test_lagged_push_and_outputs_reject_null_handles():
    import hsi_b200 as hsi
    L = hsi.cxx_lib()
    assert L.hsi_lagged_push(None, None, None) == hsi.E_INVALID
    assert L.hsi_lagged_outputs_of(None, None) == hsi.E_INVALID
    L.hsi_lagged_destroy(None)
