"""GPU: batched scene moments (hsi_scene_moments_batch).

The tensor path's partial sums are exact integers until the final FP64
rebuild, and the reference point comes from order-independent minima and
maxima, so each job's moments must equal hsi_scene_moments on that frame
alone bit for bit, whatever else shares the batch (frames of other sizes,
band counts and element types; more than the 64 frames of one launch
sequence; frames that fall back to the FP32 path).  Repeated runs must be
bit-identical too.  Accuracy against the FP64 oracle uses the tolerances of
test_gpu_stats.py (covariance within 5e-8 of its largest entry, mean 1e-7).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _frame(hsi, B, H, W, dtype, seed):
    sc = hsi.scene(B, n_targets=2, target_frac=0.01, anomaly_frac=0.005, frame_seed=seed)
    cube, _ = hsi.generate(sc, H, W, dtype=dtype)
    return cube


def _run_batch(hsi, specs, cubes, refs=None):
    outs, jobs = [], []
    for i, ((B, H, W, dt), cube) in enumerate(zip(specs, cubes)):
        out = torch.full((hsi.moments_elements(B),), float("nan"), dtype=torch.float64, device="cuda")
        ref = None if refs is None else refs[i]
        jobs.append(hsi.moments_job(cube, H, W, B, out, dtype=dt, reference=ref))
        outs.append(out)
    hsi.scene_moments_batch(jobs)
    torch.cuda.synchronize()
    return outs


def _cov_err(hsi, orc, cube, out, B, P):
    host = cube[:, :P].float().cpu().numpy().reshape(B, P)
    s0, o0, n0 = orc.moments(host)
    s, o, n = [x.cpu().numpy() for x in hsi.split_moments(out, B)]
    assert float(n) == P == n0
    mu0, mu = s0 / n0, s / n
    c0 = o0 / n0 - np.outer(mu0, mu0)
    c = o / n - np.outer(mu, mu)
    return (np.max(np.abs(c - c0)) / np.max(np.abs(c0)),
            np.max(np.abs(mu - mu0) / np.maximum(np.abs(mu0), 1e-3)))


def test_mixed_batch_equals_single_frames_bit_for_bit(hsi, orc):
    # (bands, height, width, dtype): tensor f32 / f16 frames of several sizes,
    # a small frame and a 224-band frame (FP32 path), interleaved
    specs = [(113, 256, 256, 0), (16, 200, 300, 1), (127, 181, 190, 0), (60, 64, 64, 0),
             (224, 128, 128, 0), (113, 512, 300, 1), (3, 300, 301, 0), (113, 1024, 1024, 0)]
    cubes = [_frame(hsi, B, H, W, dt, 0x5EED7000 + i) for i, (B, H, W, dt) in enumerate(specs)]
    got = _run_batch(hsi, specs, cubes)
    again = _run_batch(hsi, specs, cubes)
    for i, ((B, H, W, dt), cube) in enumerate(zip(specs, cubes)):
        single = hsi.scene_moments(cube, H, W, B, dtype=dt)
        torch.cuda.synchronize()
        assert torch.equal(got[i], single), i
        assert torch.equal(got[i], again[i]), i
        if i in (0, 1, 7):
            cov, mean = _cov_err(hsi, orc, cube, got[i], B, H * W)
            assert cov < 5e-8 and mean < 1e-7, (i, cov, mean)


def test_more_frames_than_one_launch_sequence(hsi):
    """70 tensor-path frames, 66 of them FP32: three launch sequences (64 + 2
    FP32 frames, 4 FP16 frames) on one workspace."""
    specs = [(24 + (i % 5), 180 + (i % 3), 190, 1 if i >= 66 else 0) for i in range(70)]
    cubes = [_frame(hsi, B, H, W, dt, 0x5EED7100 + i) for i, (B, H, W, dt) in enumerate(specs)]
    got = _run_batch(hsi, specs, cubes)
    for i in (0, 1, 37, 63, 64, 65, 69):
        B, H, W, dt = specs[i]
        single = hsi.scene_moments(cubes[i], H, W, B, dtype=dt)
        torch.cuda.synchronize()
        assert torch.equal(got[i], single), i


def test_out_of_range_frame_is_rerun_alone(hsi, orc):
    """One frame of the batch holds values far outside its subsample's range
    (between the sampled runs): that frame's pass is re-run with every band's
    whole-frame range, the others are not touched, and all stay accurate.
    The two bands holding the outliers get a fixed-point grid of 2^-21 of
    their range (|x - r| up to 500 here, a step of ~2.4e-4), whose rounding
    noise on the mean is ~ step / sqrt(12 N) = 1.3e-7: those bands are held to
    5x that; every other entry to the usual tolerances."""
    specs = [(113, 512, 600, 0), (113, 512, 600, 0), (113, 512, 600, 0)]
    cubes = [_frame(hsi, B, H, W, dt, 0x5EED7200 + i) for i, (B, H, W, dt) in enumerate(specs)]
    P = 512 * 600
    # frames above 512 runs of 64 pixels sample every (runs // 256)-th run,
    # here every 18th: pixels 64..1151 are never in the subsample
    cubes[1][5, 100] = 500.0
    cubes[1][70, 64] = -300.0
    got = _run_batch(hsi, specs, cubes)
    for i, ((B, H, W, dt), cube) in enumerate(zip(specs, cubes)):
        single = hsi.scene_moments(cube, H, W, B, dtype=dt)
        torch.cuda.synchronize()
        assert torch.equal(got[i], single), i
        host = cube[:, :P].float().cpu().numpy().reshape(B, P)
        s0, o0, n0 = orc.moments(host)
        s, o, n = [x.cpu().numpy() for x in hsi.split_moments(got[i], B)]
        mu0, mu = s0 / n0, s / n
        c0 = o0 / n0 - np.outer(mu0, mu0)
        c = o / n - np.outer(mu, mu)
        coarse = [5, 70] if i == 1 else []
        fine = np.setdiff1d(np.arange(B), coarse)
        scale = np.max(np.abs(c0[np.ix_(fine, fine)]))
        assert np.max(np.abs(c - c0)[np.ix_(fine, fine)]) / scale < 5e-8, i
        assert np.max(np.abs(mu - mu0)[fine] / np.maximum(np.abs(mu0[fine]), 1e-3)) < 1e-7, i
        for b in coarse:
            step = 500.0 * 2.0 ** -21 * 2
            bound = 5 * step / np.sqrt(12 * P)
            assert abs(mu[b] - mu0[b]) < bound, (b, mu[b] - mu0[b], bound)
            # covariance row of the band: its rounding noise times the other band's
            # spread, |dc_bj| ~ sigma_j * step / sqrt(12 N) (twice that on the diagonal)
            sigma = np.sqrt(np.diag(c0))
            assert np.max(np.abs(c[b] - c0[b]) / sigma) < 2 * bound, b


def test_caller_reference_and_validation(hsi, orc):
    B, H, W = 40, 200, 200
    cube = _frame(hsi, B, H, W, 0, 0x5EED7300)
    ref = cube[:, :H * W].float().mean(1).contiguous()
    got = _run_batch(hsi, [(B, H, W, 0)], [cube], refs=[ref])[0]
    single = hsi.scene_moments(cube, H, W, B, reference=ref)
    torch.cuda.synchronize()
    assert torch.equal(got, single)
    cov, mean = _cov_err(hsi, orc, cube, got, B, H * W)
    assert cov < 5e-8 and mean < 1e-7
    out = torch.empty(hsi.moments_elements(B), dtype=torch.float64, device="cuda")
    bad = hsi.moments_job(cube, H, W, 0, out)
    with pytest.raises(hsi.HsiError):
        hsi.scene_moments_batch([hsi.moments_job(cube, H, W, B, out), bad])
    small = torch.empty(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(hsi.HsiError) as e:
        hsi.scene_moments_batch([hsi.moments_job(cube, H, W, B, out)], workspace=small)
    assert e.value.status == hsi.E_WORKSPACE


def test_split_path_for_128_to_254_bands(hsi, orc):
    """Frames of 128..254 bands and at least 32768 pixels take the split path:
    two contiguous band views of at most 127 bands on the tensor cores (exact
    integer sums) and the cross block between them on the CUDA cores.  Each
    frame must meet the FP64 oracle at the tolerances above, be bit-identical
    run to run, and equal its single-frame result inside a mixed batch."""
    specs = [(224, 256, 300, 0), (113, 256, 256, 0), (224, 200, 200, 1), (254, 190, 190, 0), (128, 256, 256, 0)]
    cubes = [_frame(hsi, B, H, W, dt, 0x5EED7400 + i) for i, (B, H, W, dt) in enumerate(specs)]
    got = _run_batch(hsi, specs, cubes)
    again = _run_batch(hsi, specs, cubes)
    for i, ((B, H, W, dt), cube) in enumerate(zip(specs, cubes)):
        single = hsi.scene_moments(cube, H, W, B, dtype=dt)
        torch.cuda.synchronize()
        assert torch.equal(got[i], single), i
        assert torch.equal(got[i], again[i]), i
        cov, mean = _cov_err(hsi, orc, cube, got[i], B, H * W)
        assert cov < 5e-8 and mean < 1e-7, (i, cov, mean)


@pytest.mark.parametrize("B", [129, 201, 252, 253])
def test_split_band_counts(hsi, orc, B):
    """Odd and extreme band counts of the split paths: quarters of unequal size
    (129, 201), the largest all-tensor-core frame (252 = 4 x 63) and the first
    that keeps the CUDA-core cross block (253)."""
    H, W = 200, 170
    cube = _frame(hsi, B, H, W, 0, 0x5EED7500 + B)
    got = _run_batch(hsi, [(B, H, W, 0)], [cube])[0]
    single = hsi.scene_moments(cube, H, W, B)
    torch.cuda.synchronize()
    assert torch.equal(got, single)
    cov, mean = _cov_err(hsi, orc, cube, got, B, H * W)
    assert cov < 5e-8 and mean < 1e-7, (cov, mean)


def test_split_path_with_caller_reference(hsi, orc):
    """A caller's per-band reference points keep the two-view split form (the
    references apply to whole bands); the result is as accurate."""
    B, H, W = 224, 200, 200
    cube = _frame(hsi, B, H, W, 0, 0x5EED7600)
    ref = cube[:, :H * W].float().mean(1).contiguous()
    got = _run_batch(hsi, [(B, H, W, 0)], [cube], refs=[ref])[0]
    cov, mean = _cov_err(hsi, orc, cube, got, B, H * W)
    assert cov < 5e-8 and mean < 1e-7, (cov, mean)
