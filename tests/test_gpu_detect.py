"""GPU parity: detection compaction must be bit-exact against the reference's
detect_cpu semantics (the fixtures) and the FP64 oracle's restatement of it."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _gpu_detect(hsi, score, target, H, W, thr, r, higher, capacity=1 << 22, count0=0):
    s = torch.from_numpy(np.ascontiguousarray(score, np.float32).reshape(-1)).cuda()
    t = None if target is None else torch.from_numpy(np.ascontiguousarray(target, np.int32).reshape(-1)).cuda()
    count = torch.full((1,), count0, dtype=torch.int32, device="cuda")
    cnt, out = hsi.detect(s, t, H, W, thr, r, 1 if higher else 0, capacity, count=count)
    torch.cuda.synchronize()
    return hsi.detections_to_numpy(cnt, out, capacity + count0 if capacity else 0)


def _tuples(d):
    return [(int(r["x"]), int(r["y"]), int(r["target"]), float(r["score"])) for r in d]


def test_golden_maps(hsi, golden):
    score, which = golden["sam_best_score"], golden["sam_best_target"]
    for r in (0, 1, 2, 3):
        n, d = _gpu_detect(hsi, score, which, 24, 32, float(golden["sam_threshold"]), r, False)
        assert _tuples(d) == _tuples(golden[f"sam_detect_r{r}"])
    for r in (0, 2):
        n, d = _gpu_detect(hsi, score, which, 24, 32, float(golden["sam_threshold_hi"]), r, True)
        assert _tuples(d) == _tuples(golden[f"sam_detect_hi_r{r}"])


def test_golden_hand_built_cases(hsi, golden):
    z = None
    for r in (0, 2):
        n, d = _gpu_detect(hsi, golden["case_blob_score"], z, 9, 9, 0.1, r, False)
        assert _tuples(d) == _tuples(golden[f"case_blob_detect_r{r}"])
    n, d = _gpu_detect(hsi, golden["case_plateau_score"], z, 5, 5, 0.1, 2, False)
    assert _tuples(d) == _tuples(golden["case_plateau_detect"])
    n, d = _gpu_detect(hsi, golden["case_polarity_score"], z, 7, 7, 0.1, 1, False)
    assert _tuples(d) == _tuples(golden["case_polarity_low"])
    n, d = _gpu_detect(hsi, golden["case_polarity_score"], z, 7, 7, 0.9, 1, True)
    assert _tuples(d) == _tuples(golden["case_polarity_high"])
    n, d = _gpu_detect(hsi, golden["case_extremum_score"], z, 9, 9, 0.55, 3, True)
    assert _tuples(d) == _tuples(golden["case_extremum_high"])


@pytest.mark.parametrize("shape", [(1, 1), (1, 700), (700, 1), (37, 53), (256, 256), (130, 300), (1024, 2048)])
@pytest.mark.parametrize("radius", [0, 1, 2, 4, 8, 11])
@pytest.mark.parametrize("higher", [False, True])
def test_random_plateaus_bit_exact(hsi, orc, shape, radius, higher):
    H, W = shape
    rng = np.random.default_rng(H * 7 + W + radius)
    # quantised values make many exact ties, exercising the index tie-break
    score = (rng.integers(0, 40, H * W) / 40.0).astype(np.float32)
    target = rng.integers(0, 8, H * W).astype(np.int32)
    thr = 0.9 if higher else 0.1
    n0, want = orc.detect(score, target, H, W, thr, radius, higher, capacity=1 << 22)
    n, got = _gpu_detect(hsi, score, target, H, W, thr, radius, higher)
    assert n == n0 <= 1 << 22
    assert _tuples(got) == _tuples(want)


@pytest.mark.parametrize("radius", [1, 3, 4])
@pytest.mark.parametrize("higher", [False, True])
def test_sparse_and_dense_segments_bit_exact(hsi, orc, radius, higher):
    """Rows alternate between few candidates and many, in a map three row
    segments wide with a ragged last segment, so tiles see both densities
    within one window."""
    H, W = 96, 4500
    rng = np.random.default_rng(1000 + radius)
    q = rng.integers(0, 50, (H, W)) / 50.0
    sparse_rows = (np.arange(H) // 3) % 2 == 0
    # sparse rows: candidates only where a rare draw lifts the score past the threshold
    rare = rng.random((H, W)) < 0.002
    q[sparse_rows] = np.where(rare[sparse_rows], 0.98, q[sparse_rows] * 0.5)
    score = (q if higher else 1.0 - q).astype(np.float32)
    target = rng.integers(0, 8, H * W).astype(np.int32)
    thr = 0.9 if higher else 0.1
    n0, want = orc.detect(score.reshape(-1), target, H, W, thr, radius, higher, capacity=1 << 22)
    n, got = _gpu_detect(hsi, score.reshape(-1), target, H, W, thr, radius, higher)
    assert n == n0
    assert _tuples(got) == _tuples(want)


def test_capacity_overflow_keeps_raster_prefix(hsi, orc):
    H, W = 300, 301
    rng = np.random.default_rng(5)
    score = rng.uniform(0, 1, H * W).astype(np.float32)
    n0, want = orc.detect(score, None, H, W, 0.2, 0, False)
    cap = 1000
    assert n0 > cap
    n, got = _gpu_detect(hsi, score, None, H, W, 0.2, 0, False, capacity=cap)
    assert n == n0
    assert _tuples(got[:cap]) == _tuples(want[:cap])


def test_count_offset_and_nan(hsi, orc):
    score = np.array([0.05, np.nan, 0.01, 0.5, np.nan, 0.02], np.float32)
    n0, want = orc.detect(score, None, 1, 6, 0.1, 0, False)
    s = torch.from_numpy(score).cuda()
    count = torch.full((1,), 5, dtype=torch.int32, device="cuda")
    out = torch.full((16, 4), -1, dtype=torch.int32, device="cuda")
    cnt, out = hsi.detect(s, None, 1, 6, 0.1, 0, 0, 16, out=out, count=count)
    torch.cuda.synchronize()
    assert int(cnt.item()) == 5 + n0 == 8
    o = out.cpu().numpy()
    assert (o[:5] == -1).all()
    dt = np.dtype([("x", "<i4"), ("y", "<i4"), ("target", "<i4"), ("score", "<f4")])
    assert _tuples(o[5:8].copy().view(dt).reshape(-1)) == _tuples(want)


def test_workspace_is_checked(hsi):
    s = torch.zeros(64, device="cuda")
    small = torch.empty(8, dtype=torch.uint8, device="cuda")
    with pytest.raises(hsi.HsiError) as e:
        hsi.detect(s, None, 8, 8, 0.1, 0, 0, 16, workspace=small)
    assert e.value.status == hsi.E_WORKSPACE


def test_batched_maps_match_single_calls(hsi, orc):
    """Up to 64 maps of different sizes, radii and polarities in one call."""
    rng = np.random.default_rng(77)
    specs = [(37, 53, 0, False), (1, 1, 2, True), (64, 2100, 2, False), (300, 7, 4, True), (128, 128, 6, False),
             (5, 5000, 1, True)]
    jobs, keep = [], []
    for (H, W, r, higher) in specs:
        score = (rng.integers(0, 30, H * W) / 30.0).astype(np.float32)
        target = rng.integers(0, 8, H * W).astype(np.int32)
        s = torch.from_numpy(score).cuda()
        t = torch.from_numpy(target).cuda()
        out = torch.full((H * W + 1, 4), -1, dtype=torch.int32, device="cuda")
        count = torch.zeros(1, dtype=torch.int32, device="cuda")
        thr = 0.85 if higher else 0.15
        jobs.append(hsi.detect_job(s, t, H, W, thr, r, 1 if higher else 0, H * W + 1, out, count))
        keep.append((score, target, H, W, thr, r, higher, s, t, out, count))
    ws = torch.empty(hsi.detect_batch_workspace_bytes(jobs), dtype=torch.uint8, device="cuda")
    hsi.detect_batch(jobs, ws)
    torch.cuda.synchronize()
    for score, target, H, W, thr, r, higher, _, _, out, count in keep:
        n0, want = orc.detect(score, target, H, W, thr, r, higher, capacity=H * W + 1)
        n, got = hsi.detections_to_numpy(count, out, H * W + 1)
        assert n == n0
        assert _tuples(got) == _tuples(want)


@pytest.mark.parametrize("shape", [(1, 4), (3, 508), (65, 512), (66, 516), (129, 1028)])
@pytest.mark.parametrize("radius", [-1, 3, 4, 5])
@pytest.mark.parametrize("higher", [False, True])
def test_tile_edges_and_kernel_switch_bit_exact(hsi, orc, shape, radius, higher):
    """Widths that are multiples of 4 around the 512-column tiles and 64-row bands of the
    four-column flags kernel, at radii on both sides of its limit (4; 5 takes the plain
    kernel), with NaN scores and quantised ties."""
    H, W = shape
    rng = np.random.default_rng(H * 131 + W * 7 + radius + 3)
    score = (rng.integers(0, 25, H * W) / 25.0).astype(np.float32)
    score[rng.integers(0, H * W, max(1, H * W // 40))] = np.nan
    target = rng.integers(0, 8, H * W).astype(np.int32)
    thr = 0.88 if higher else 0.12
    n0, want = orc.detect(score, target, H, W, thr, radius, higher, capacity=1 << 22)
    n, got = _gpu_detect(hsi, score, target, H, W, thr, radius, higher)
    assert n == n0
    assert _tuples(got) == _tuples(want)


def test_unaligned_map_takes_the_plain_kernel(hsi, orc):
    """A map that does not start on 16 bytes runs the plain flags kernel, with the same result."""
    H, W, r = 70, 260, 2
    rng = np.random.default_rng(91)
    score = (rng.integers(0, 25, H * W) / 25.0).astype(np.float32)
    target = rng.integers(0, 8, H * W).astype(np.int32)
    buf = torch.zeros(H * W + 4, device="cuda")
    buf[1:1 + H * W] = torch.from_numpy(score).cuda()
    s = buf[1:1 + H * W]
    assert s.data_ptr() % 16 == 4
    t = torch.from_numpy(target).cuda()
    for higher in (False, True):
        thr = 0.88 if higher else 0.12
        n0, want = orc.detect(score, target, H, W, thr, r, higher, capacity=1 << 16)
        cnt, out = hsi.detect(s, t, H, W, thr, r, 1 if higher else 0, 1 << 16)
        torch.cuda.synchronize()
        n, got = hsi.detections_to_numpy(cnt, out, 1 << 16)
        assert n == n0
        assert _tuples(got) == _tuples(want)
