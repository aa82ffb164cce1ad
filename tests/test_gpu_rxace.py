"""GPU parity: RX and ACE against the FP64 oracle, and the error the device-built
statistics add to every score map.

Tolerances (stated here): RX relative |gpu - fp64| / max(1, |fp64|) <= 1e-4
(tests/test_detector.cpp:126 convention); ACE and CEM absolute <= 1e-4; best-
target labels may differ only where the two targets' oracle ACE values are
within 1e-4.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _download(cube, B, P):
    return cube[:, :P].float().cpu().numpy().reshape(B, P)


def _scene(hsi, H, W, B, T, seed, dtype=0):
    sc = hsi.scene(B, n_targets=T, target_frac=0.002, anomaly_frac=0.001, library_seed=0x5EED2000 + B,
                   frame_seed=seed)
    cube, truth = hsi.generate(sc, H, W, dtype=dtype)
    return cube, truth, hsi.scene_targets(sc)


def _fp64_stats(orc, host, lib, loading):
    s, o, n = orc.moments(host)
    st, S = orc.build_statistics(s, o, n, lib, loading)
    assert st == 0
    return S


def _pack(S):
    return np.concatenate([S["mean"], S["whitener"].reshape(-1), S["target_white"].reshape(-1), S["target_norm2"],
                           S["cem_weight"].reshape(-1)])


def _check_scores(orc, host, S, rx, ace, at, maps, T):
    best0, w0, rx0, all0 = orc.ace(host, S)
    rx_err = np.max(np.abs(rx - rx0) / np.maximum(1.0, np.abs(rx0)))
    assert rx_err <= TOL, f"RX relative error {rx_err:.3e}"
    if maps is not None:
        assert np.max(np.abs(maps - all0)) <= TOL
    assert np.max(np.abs(ace - best0)) <= TOL, f"ACE error {np.max(np.abs(ace - best0)):.3e}"
    for p in np.nonzero(at != w0)[0]:
        g = at[p]
        assert g >= 0 and abs(all0[g, p] - best0[p]) <= TOL
    return rx_err


@pytest.mark.parametrize("simt", [True, False])
@pytest.mark.parametrize("B,T", [(16, 3), (113, 8), (127, 1), (113, 16), (224, 16)])
def test_rx_ace_with_fp64_statistics(hsi, orc, simt, B, T):
    """simt=False is the tensor-core path (INT8 limbs); (113, 16) takes two
    target passes there (15 + 1 targets), the best carried between them."""
    if not simt and B > 127:
        pytest.skip("the tensor-core path holds at most 127 bands")
    H, W = 96, 80
    cube, _, lib = _scene(hsi, H, W, B, T, seed=B * 7 + T)
    P = H * W
    host = _download(cube, B, P)
    S = _fp64_stats(orc, host, lib, 1e-5)
    stats = torch.from_numpy(_pack(S)).cuda()
    rx = torch.zeros(P, device="cuda")
    ace = torch.zeros(P, device="cuda")
    at = torch.zeros(P, dtype=torch.int32, device="cuda")
    maps = torch.zeros((T, P), device="cuda")
    hsi.rx_ace(cube, H, W, B, stats, T, rx=rx, ace_best=ace, ace_target=at, ace_maps=maps, simt=simt)
    torch.cuda.synchronize()
    _check_scores(orc, host, S, rx.cpu().numpy(), ace.cpu().numpy(), at.cpu().numpy(), maps.cpu().numpy(), T)


@pytest.mark.parametrize("dtype", [0, 1])
def test_rx_ace_tensor_core_at_size(hsi, orc, dtype):
    """512 x 512 x 113 with anomalies, 8 targets, both cube types: the tensor-core
    path against the FP64 oracle on the same (device-read-back) cube."""
    H, W, B, T = 512, 512, 113, 8
    cube, _, lib = _scene(hsi, H, W, B, T, seed=0x5EED2001, dtype=dtype)
    P = H * W
    host = _download(cube, B, P)
    S = _fp64_stats(orc, host, lib, 1e-6)
    stats = torch.from_numpy(_pack(S)).cuda()
    rx = torch.zeros(P, device="cuda")
    ace = torch.zeros(P, device="cuda")
    at = torch.zeros(P, dtype=torch.int32, device="cuda")
    maps = torch.zeros((T, P), device="cuda")
    hsi.rx_ace(cube, H, W, B, stats, T, dtype=dtype, rx=rx, ace_best=ace, ace_target=at, ace_maps=maps, simt=False)
    torch.cuda.synchronize()
    _check_scores(orc, host, S, rx.cpu().numpy(), ace.cpu().numpy(), at.cpu().numpy(), maps.cpu().numpy(), T)


def test_rx_ace_tensor_core_rejects_too_many_bands(hsi):
    cube = torch.zeros((128, 64), device="cuda")
    stats = torch.zeros(128 + 128 * 128, dtype=torch.float64, device="cuda")
    with pytest.raises(hsi.HsiError):
        hsi.rx_ace(cube, 8, 8, 128, stats, 0, rx=torch.zeros(64, device="cuda"), simt=False)


@pytest.mark.parametrize("simt", [True, False])
def test_rx_ace_reference_properties(hsi, orc, simt):
    """RX ranks planted anomalies above the background, ACE peaks on its own
    target (tests/test_detectors.cpp:82-184), on the GPU path."""
    H, W, B = 40, 48, 14
    rng = np.random.default_rng(3)
    P = H * W
    t = np.arange(B, dtype=np.float32) / B
    a = rng.standard_normal(P).astype(np.float32) * 0.05
    bb = rng.standard_normal(P).astype(np.float32) * 0.03
    host = (0.30 + 0.15 * t[:, None] + a[None] * (t * (1 - t))[:, None] + bb[None] * np.sin(4 * t)[:, None]
            + rng.standard_normal((B, P)) * 0.01).astype(np.float32)
    anomaly = (0.75 - 0.55 * t).astype(np.float32)
    idx = [P // 7, P // 3, (2 * P) // 3]
    for p in idx:
        host[:, p] = anomaly + rng.standard_normal(B).astype(np.float32) * 0.01
    lib = np.stack([anomaly, (0.30 + 0.15 * t).astype(np.float32)])
    stride = hsi.plane_stride(H, W)
    cube = torch.zeros((B, stride), device="cuda")
    cube[:, :P] = torch.from_numpy(host).cuda()
    gm = hsi.scene_moments(cube, H, W, B)
    s64, _, status = hsi.build_statistics(gm, B, torch.from_numpy(lib).cuda(), loading=1e-6)
    rx = torch.zeros(P, device="cuda")
    ace = torch.zeros(P, device="cuda")
    at = torch.zeros(P, dtype=torch.int32, device="cuda")
    hsi.rx_ace(cube, H, W, B, s64[0], 2, rx=rx, ace_best=ace, ace_target=at, simt=simt)
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    rx, ace, at = rx.cpu().numpy(), ace.cpu().numpy(), at.cpu().numpy()
    assert rx[idx].min() > np.delete(rx, idx).max()
    assert ace.min() >= 0 and ace.max() <= 1
    assert (ace[idx] >= 0.9).all() and (at[idx] == 0).all()


@pytest.mark.parametrize("simt_moments", [False, True])
def test_device_statistics_error_budget(hsi, orc, simt_moments):
    """Moments and factorisation on the device; scores computed by the FP64
    oracle with those statistics.  Isolates the error the statistics add."""
    H, W, B, T = 512, 512, 113, 8
    cube, _, lib = _scene(hsi, H, W, B, T, seed=0x5EED2001)
    P = H * W
    host = _download(cube, B, P)
    S0 = _fp64_stats(orc, host, lib, 1e-6)
    gm = hsi.scene_moments(cube, H, W, B, simt=simt_moments)
    s64, _, status = hsi.build_statistics(gm, B, torch.from_numpy(lib).cuda(), loading=1e-6)
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    S = hsi.unpack_statistics(s64[0].cpu().numpy(), B, T)
    rx0 = orc.rx(host, S0).astype(np.float64)
    rx = orc.rx(host, S).astype(np.float64)
    assert np.max(np.abs(rx - rx0) / np.maximum(1.0, rx0)) <= TOL
    a0 = orc.ace(host, S0)[3]
    a = orc.ace(host, S)[3]
    assert np.max(np.abs(a - a0)) <= TOL
    c0 = orc.cem(host, S0)[2]
    c = orc.cem(host, S)[2]
    assert np.max(np.abs(c - c0)) <= TOL
