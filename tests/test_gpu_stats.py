"""GPU parity: scene moments (tensor-core and SIMT paths) and the FP64
factorisation against the FP64 oracle and the reference's own fixtures.

Tolerances (stated here):
  moments      : count exact; mean relative error < 1e-7; covariance entries
                 within 5e-8 of the largest covariance entry (RX/ACE amplify
                 covariance errors by the condition number, ~4000 here);
  statistics   : from the same FP64 moments, every FP64 statistic within
                 1e-9 relative (different order of FP64 operations);
  RX           : |gpu - fp64| / max(1, |fp64|) <= 1e-4  (the reference's
                 relative convention, tests/test_detector.cpp:126);
  ACE, CEM     : absolute error <= 1e-4.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _download(cube, B, P):
    return cube[:, :P].float().cpu().numpy().reshape(B, P)


def _cov(s, o, n):
    mu = s / n
    return o / n - np.outer(mu, mu), mu


def _check_moments(hsi, orc, host, gm, B, P, cov_tol=5e-8, mean_tol=1e-7):
    s0, o0, n0 = orc.moments(host)
    s, o, n = [x.cpu().numpy() for x in hsi.split_moments(gm, B)]
    assert float(n) == P == n0
    c0, mu0 = _cov(s0, o0, n0)
    c, mu = _cov(s, o, float(n))
    assert np.max(np.abs(mu - mu0) / np.maximum(np.abs(mu0), 1e-3)) < mean_tol
    scale = np.max(np.abs(c0))
    err = np.max(np.abs(c - c0)) / max(scale, 1e-30)
    assert err < cov_tol, f"covariance error {err:.3e} of max entry"
    assert np.allclose(o, o.T, rtol=0, atol=0)
    return err


@pytest.mark.parametrize("path", [None, "simt", "tc"])
@pytest.mark.parametrize("B", [1, 3, 16, 113, 127, 128, 224, 254, 255])
@pytest.mark.parametrize("shape", [(7, 13), (64, 64), (256, 300)])
def test_moments_match_fp64(hsi, orc, path, B, shape):
    H, W = shape
    if path == "tc" and B > 127:
        pytest.skip("tensor-core path holds at most 127 bands")
    sc = hsi.scene(B, n_targets=2, target_frac=0.01, anomaly_frac=0.005, frame_seed=B * 31 + H)
    cube, _ = hsi.generate(sc, H, W)
    host = _download(cube, B, H * W)
    gm = hsi.scene_moments(cube, H, W, B, path=path)
    torch.cuda.synchronize()
    # the forced integer path on tiny frames: its zero-mean residue shrinks as 1/sqrt(N)
    small = 1.0 / np.sqrt(H * W / 100.0)
    tol = max(5e-8, 1e-6 * small) if path == "tc" else 5e-8
    mtol = max(1e-7, 1e-6 * small) if path == "tc" else 1e-7
    _check_moments(hsi, orc, host, gm, B, H * W, cov_tol=tol, mean_tol=mtol)


@pytest.mark.parametrize("dtype", [0, 1])
def test_moments_fp16_cube(hsi, orc, dtype):
    H, W, B = 128, 96, 113
    sc = hsi.scene(B, n_targets=4, target_frac=0.01, frame_seed=5)
    cube, _ = hsi.generate(sc, H, W, dtype=dtype)
    host = _download(cube, B, H * W)
    gm = hsi.scene_moments(cube, H, W, B, dtype=dtype)
    torch.cuda.synchronize()
    _check_moments(hsi, orc, host, gm, B, H * W)


def test_moments_with_given_reference(hsi, orc):
    H, W, B = 64, 80, 113
    sc = hsi.scene(B, n_targets=1, frame_seed=9)
    cube, _ = hsi.generate(sc, H, W)
    host = _download(cube, B, H * W)
    for ref in (np.zeros(B, np.float32), host.mean(axis=1).astype(np.float32) * 1.1):
        gm = hsi.scene_moments(cube, H, W, B, reference=torch.from_numpy(ref).cuda())
        torch.cuda.synchronize()
        if ref.any():
            _check_moments(hsi, orc, host, gm, B, H * W)
        else:
            # no shift: the sums are still exact enough for the correlation
            s0, o0, n0 = orc.moments(host)
            o = hsi.split_moments(gm, B)[1].cpu().numpy()
            assert np.max(np.abs(o - o0)) / np.max(np.abs(o0)) < 1e-6


def test_moments_are_deterministic(hsi):
    H, W, B = 200, 200, 113
    cube, _ = hsi.generate(hsi.scene(B, frame_seed=3), H, W)
    a = hsi.scene_moments(cube, H, W, B).cpu().numpy()
    b = hsi.scene_moments(cube, H, W, B).cpu().numpy()
    assert np.array_equal(a, b)


def _fp64_moments_on_device(orc, host):
    s, o, n = orc.moments(host)
    return torch.from_numpy(np.concatenate([s, o.reshape(-1), [n]])).cuda(), (s, o, n)


# 129..238 bands: one packed triangle in shared memory turned into L and then W
# in place (224: the inverse's block-row buffer in shared memory too; 225 and
# 238: in the workspace); 239 and 254: the matrices in the workspace.
@pytest.mark.parametrize("B,T", [(12, 2), (113, 8), (128, 16), (129, 4), (176, 3), (224, 16), (225, 16), (238, 5),
                                 (239, 2), (254, 16)])
def test_factor_matches_fp64_oracle(hsi, orc, B, T):
    H, W = 48, 64
    sc = hsi.scene(B, n_targets=T, target_frac=0.01, frame_seed=B + T)
    cube, _ = hsi.generate(sc, H, W)
    host = _download(cube, B, H * W)
    lib = hsi.scene_targets(sc)
    gm, (s, o, n) = _fp64_moments_on_device(orc, host)
    s64, s32, status = hsi.build_statistics(gm, B, torch.from_numpy(lib).cuda(), loading=1e-5, want32=True)
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    st, want = orc.build_statistics(s, o, n, lib, 1e-5)
    assert st == 0
    got = hsi.unpack_statistics(s64[0].cpu().numpy(), B, T)
    for k in ("mean", "whitener", "target_white", "target_norm2", "cem_weight"):
        ref = want[k]
        err = np.max(np.abs(got[k] - ref)) / max(np.max(np.abs(ref)), 1e-30)
        assert err < 1e-9, f"{k}: {err:.3e}"
    assert np.all(np.triu(got["whitener"], 1) == 0)
    g32 = hsi.unpack_statistics(s32[0].cpu().numpy(), B, T)
    np.testing.assert_array_equal(g32["whitener"], got["whitener"].astype(np.float32))


def test_factor_against_reference_fixtures(hsi, golden):
    for prefix in ("stats", "b113"):
        g = lambda k: golden[f"{prefix}_{k}"]  # noqa: E731
        B = g("sum").shape[0]
        lib = g("library")
        T = lib.shape[0]
        m = torch.from_numpy(np.concatenate([g("sum"), g("outer").reshape(-1), [float(g("count"))]])).cuda()
        # the fixtures hold the lower triangle only (SpectralMoments layout); mirror it
        o = np.tril(g("outer")) + np.tril(g("outer"), -1).T
        m = torch.from_numpy(np.concatenate([g("sum"), o.reshape(-1), [float(g("count"))]])).cuda()
        _, s32, status = hsi.build_statistics(m, B, torch.from_numpy(lib).cuda(), loading=float(g("loading")),
                                              want64=False, want32=True)
        torch.cuda.synchronize()
        assert int(status[0]) == 0
        got = hsi.unpack_statistics(s32[0].cpu().numpy(), B, T)
        for k in ("mean", "whitener", "target_white", "target_norm2", "cem_weight"):
            ref = g(k)
            err = np.max(np.abs(got[k] - ref)) / max(np.max(np.abs(ref)), 1e-30)
            assert err < 1e-5, f"{prefix} {k}: {err:.3e}"


def test_factor_reports_singular_and_empty(hsi, orc, golden):
    host = golden["singular_cube"].reshape(4, -1)
    s, o, n = orc.moments(host)
    m = torch.from_numpy(np.concatenate([s, o.reshape(-1), [n]])).cuda()
    _, _, st0 = hsi.build_statistics(m, 4, None, loading=0.0)
    _, _, st1 = hsi.build_statistics(m, 4, None, loading=1e-3)
    empty = torch.zeros(4 + 16 + 1, dtype=torch.float64, device="cuda")
    _, _, st2 = hsi.build_statistics(empty, 4, None, loading=1e-3)
    torch.cuda.synchronize()
    assert int(st0[0]) == hsi.E_NOT_POSITIVE_DEFINITE
    assert int(st1[0]) == 0
    assert int(st2[0]) == hsi.E_EMPTY
    assert "loading" in hsi.status_string(hsi.E_NOT_POSITIVE_DEFINITE)


def test_batched_factor(hsi, orc):
    B, T, F = 113, 8, 5
    ms, libs, wants = [], [], []
    for f in range(F):
        sc = hsi.scene(B, n_targets=T, target_frac=0.01, frame_seed=100 + f, library_seed=200 + f)
        cube, _ = hsi.generate(sc, 32, 40)
        host = _download(cube, B, 32 * 40)
        lib = hsi.scene_targets(sc)
        s, o, n = orc.moments(host)
        ms.append(np.concatenate([s, o.reshape(-1), [n]]))
        libs.append(lib)
        wants.append(orc.build_statistics(s, o, n, lib, 1e-5)[1])
    m = torch.from_numpy(np.stack(ms)).cuda()
    L = torch.from_numpy(np.stack(libs)).cuda()
    s64, _, status = hsi.build_statistics(m, B, L, loading=1e-5)
    torch.cuda.synchronize()
    assert (status.cpu().numpy() == 0).all()
    for f in range(F):
        got = hsi.unpack_statistics(s64[f].cpu().numpy(), B, T)
        for k in ("whitener", "cem_weight", "target_norm2"):
            assert np.max(np.abs(got[k] - wants[f][k])) / np.max(np.abs(wants[f][k])) < 1e-9


@pytest.mark.parametrize("dtype", [0, 1])
def test_cem_end_to_end_against_fp64(hsi, orc, dtype):
    """Moments (tensor cores) -> FP64 factor -> fused SAM/CEM scoring, all on the
    device, against the FP64 oracle run on the same cube."""
    H, W, B, T = 128, 128, 113, 8
    sc = hsi.scene(B, n_targets=T, target_frac=0.002, frame_seed=0x5EED1001, library_seed=0x5EED1000)
    cube, _ = hsi.generate(sc, H, W, dtype=dtype)
    P = H * W
    host = _download(cube, B, P)
    lib = hsi.scene_targets(sc)
    tg = torch.from_numpy(lib).cuda()
    gm = hsi.scene_moments(cube, H, W, B, dtype=dtype)
    cem_w = torch.zeros((T, B), device="cuda")
    _, _, status = hsi.build_statistics(gm, B, tg, loading=1e-6, want64=False, cem_weights=cem_w)
    maps = torch.zeros((T, P), device="cuda")
    best = torch.zeros(P, device="cuda")
    bt = torch.zeros(P, dtype=torch.int32, device="cuda")
    f = hsi.make_frame(cube, H, W, B, dtype, cem_weights=cem_w, cem_maps=maps, cem_best=best, cem_best_target=bt,
                       map_stride=P)
    hsi.score_frames([f])
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    s, o, n = orc.moments(host)
    st, S = orc.build_statistics(s, o, n, lib, 1e-6)
    b0, w0, all0 = orc.cem(host, S)
    err = np.max(np.abs(maps.cpu().numpy() - all0))
    assert err <= 1e-4, f"CEM max abs error vs FP64 {err:.3e}"
