"""GPU: the integer-limb moments stay exact when the frame's range exceeds
what the subsample predicted (the conditional re-run with the observed range),
and for large offsets / gains of the data."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _check(hsi, cube, H, W, B, tol=5e-8, mean_tol=1e-7):
    P = H * W
    host = cube[:, :P].float().cpu().numpy()
    gm = hsi.scene_moments(cube, H, W, B, path="tc")
    torch.cuda.synchronize()
    s, o, n = [x.cpu().numpy() for x in hsi.split_moments(gm, B)]
    mu = s / n
    c = o / n - np.outer(mu, mu)
    # FP64 two-pass reference (mean, then centred products): the raw FP64 sums
    # of the oracle (as the reference's CPU accumulation) lose ~sqrt(N) eps of
    # sum(x^2) ~ 1e10 at a +500 offset, which is itself 3e-7 of the covariance.
    x64 = host.astype(np.float64)
    n0 = float(P)
    mu0 = x64.mean(axis=1)
    xc = x64 - mu0[:, None]
    c0 = (xc @ xc.T) / n0
    err = np.max(np.abs(c - c0)) / np.max(np.abs(c0))
    assert float(n) == n0
    assert np.max(np.abs(mu - mu0) / np.maximum(np.abs(mu0), 1e-6)) < mean_tol
    assert err < tol, f"covariance error {err:.3e}"


def test_outlier_outside_the_subsample_triggers_exact_rerun(hsi):
    H, W, B = 256, 512, 64
    cube, _ = hsi.generate(hsi.scene(B, frame_seed=11), H, W)
    # a few pixels far outside anything the subsample saw (not on its sampled runs)
    for p in (64 * 3 + 5, 64 * 700 + 9, H * W - 3):
        cube[:, p] = 40.0
    # The re-run covers the observed range (2x headroom).  With outliers ~800x
    # the typical deviation the fixed-point step grows to ~6e-5, and the
    # rounding residues leave errors of order step * sigma / sqrt(N): ~5e-7 of
    # the mean, ~2e-6 of the (outlier-dominated) largest covariance entry.
    _check(hsi, cube, H, W, B, tol=5e-6, mean_tol=2e-6)


@pytest.mark.parametrize("gain,offset", [(1000.0, 0.0), (1e-3, 0.0), (1.0, 500.0)])
def test_radiometric_scale_and_offset(hsi, gain, offset):
    H, W, B = 192, 256, 113
    cube, _ = hsi.generate(hsi.scene(B, frame_seed=12), H, W)
    cube.mul_(gain).add_(offset)
    _check(hsi, cube, H, W, B, tol=1e-7 if offset else 5e-8)
