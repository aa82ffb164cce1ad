"""GPU: hsi_detect_noalloc, the detection entry point for callers that cannot
allocate device memory (for example a plug-in whose host application hands it
only input and output buffers and owns all device memory, so it has no
workspace to pass to hsi_detect).  It keeps its scratch in an array inside
the library instead.

The lists must equal those of hsi_detect bit for bit (detection lists are
integer/index work: no tolerance), on two calls in a row with different maps,
so that whatever the first call leaves in the shared array cannot leak into
the second.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _noalloc(hsi, score, target, H, W, thr, radius, polarity, capacity):
    out = torch.full((capacity, 4), -7, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = hsi.lib().hsi_detect_noalloc(C.c_void_p(score.data_ptr()),
                                      None if target is None else C.c_void_p(target.data_ptr()), H, W,
                                      C.c_float(thr), radius, polarity, capacity, C.c_void_p(out.data_ptr()),
                                      C.c_void_p(count.data_ptr()), None)
    assert st == 0, hsi.status_string(st)
    return count, out


def _lists(count, out, capacity):
    n = int(count.item())
    return n, out[:min(n, capacity)].cpu().numpy()


@pytest.mark.parametrize("H,W,radius,polarity,thr", [
    (1024, 1024, 2, 0, 0.05),     # SAM-like: lower is better, staged NMS window
    (517, 3001, 0, 1, 0.93),      # ragged width (two segments per row), no NMS, higher is better
    (64, 4096, 5, 1, 0.90),       # radius beyond the staged tile: global-memory NMS
])
def test_noalloc_matches_hsi_detect_on_consecutive_calls(hsi, H, W, radius, polarity, thr):
    g = torch.Generator(device="cuda").manual_seed(H * 7 + W)
    capacity = 1 << 16
    for call in range(2):
        score = torch.rand((H, W), generator=g, device="cuda")
        # quantised scores make exact ties that the index tie-break must settle
        score = torch.round(score * 512) / 512
        target = torch.randint(0, 16, (H, W), generator=g, device="cuda", dtype=torch.int32)
        want_count, want_out = hsi.detect(score, target, H, W, thr, radius, polarity, capacity)
        got_count, got_out = _noalloc(hsi, score, target, H, W, thr, radius, polarity, capacity)
        torch.cuda.synchronize()
        n0, l0 = _lists(want_count, want_out, capacity)
        n1, l1 = _lists(got_count, got_out, capacity)
        assert n0 > 0, "the case should produce detections"
        assert n1 == n0, f"call {call}: count {n1} != {n0}"
        assert np.array_equal(l1, l0), f"call {call}: lists differ"


def test_noalloc_counts_past_capacity_like_hsi_detect(hsi):
    H, W, capacity = 300, 500, 1000
    score = torch.rand((H, W), device="cuda")
    want_count, want_out = hsi.detect(score, None, H, W, 0.2, 0, 0, capacity)
    got_count, got_out = _noalloc(hsi, score, None, H, W, 0.2, 0, 0, capacity)
    torch.cuda.synchronize()
    assert int(got_count.item()) == int(want_count.item()) > capacity
    assert np.array_equal(got_out.cpu().numpy(), want_out[:capacity].cpu().numpy())


def test_noalloc_rejects_maps_beyond_its_limit(hsi):
    L = hsi.lib()
    score = torch.zeros(16, device="cuda")
    out = torch.zeros((4, 4), dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    args = (C.c_void_p(score.data_ptr()), None)
    tail = (C.c_float(0.5), 0, 0, 4, C.c_void_p(out.data_ptr()), C.c_void_p(count.data_ptr()), None)
    # 8193 rows of one segment, and 4097 rows of two segments, exceed 8192 segments
    assert L.hsi_detect_noalloc(*args, 8193, 2048, *tail) == hsi.E_CAPACITY
    assert L.hsi_detect_noalloc(*args, 4097, 4096, *tail) == hsi.E_CAPACITY
    assert L.hsi_detect_noalloc(*args, 0, 16, *tail) == hsi.E_INVALID
    assert int(count.item()) == 0
