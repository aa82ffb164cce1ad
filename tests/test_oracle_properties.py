"""The reference's property tests (tests/test_sam.cpp, tests/test_detectors.cpp,
tests/test_detector.cpp, tests/test_linalg.cpp), restated against the FP64
oracle.  The same properties are replayed on the GPU path in test_gpu_*.py."""
import numpy as np
import pytest


def test_scale_invariance(orc):
    rng = np.random.default_rng(7)
    t = rng.uniform(0.05, 1.0, (1, 16)).astype(np.float32)
    px = rng.uniform(0.05, 1.0, 16).astype(np.float32)
    base, _ = orc.sam_best(px.reshape(16, 1), t)
    for gain in (0.01, 0.5, 3.0, 250.0):
        s, _ = orc.sam_best((px * np.float32(gain)).reshape(16, 1), t)
        assert abs(s[0] - base[0]) < 1e-4


def test_best_match_agrees_with_per_target_maps(orc):
    rng = np.random.default_rng(3)
    cube = rng.uniform(0, 1, (20, 50)).astype(np.float32)
    t = rng.uniform(0, 1, (5, 20)).astype(np.float32)
    s, w = orc.sam_best(cube, t)
    allm = orc.sam_all(cube, t)
    np.testing.assert_array_equal(s, allm.min(axis=0))
    np.testing.assert_array_equal(w, allm.argmin(axis=0))


def _scene(h, w, bands, seed):
    rng = np.random.default_rng(seed)
    P = h * w
    t = np.arange(bands, dtype=np.float32) / np.float32(bands)
    a = rng.standard_normal(P).astype(np.float32) * 0.05
    b = rng.standard_normal(P).astype(np.float32) * 0.03
    cube = (0.30 + 0.15 * t[:, None] + a[None] * (t * (1 - t))[:, None] + b[None] * np.sin(4 * t)[:, None]
            + rng.standard_normal((bands, P)) * 0.01).astype(np.float32)
    anomaly = (0.75 - 0.55 * t).astype(np.float32)
    idx = [P // 7, P // 3, (2 * P) // 3]
    for p in idx:
        cube[:, p] = anomaly + rng.standard_normal(bands).astype(np.float32) * 0.01
    return cube, idx, anomaly


def test_rx_ranks_anomalies_and_matches_chi_squared(orc):
    cube, idx, _ = _scene(40, 48, 16, 1)
    s, o, n = orc.moments(cube)
    st, S = orc.build_statistics(s, o, n, None, 1e-6)
    assert st == orc.STATS_OK
    rx = orc.rx(cube, S)
    bg = np.delete(rx, idx)
    assert rx[idx].min() > bg.max()
    cube, idx, _ = _scene(60, 60, 12, 2)
    s, o, n = orc.moments(cube)
    st, S = orc.build_statistics(s, o, n, None, 1e-9)
    m = np.delete(orc.rx(cube, S), idx).mean()
    assert 12 * 0.80 < m < 12 * 1.05


def test_ace_bounded_and_cem_unit_gain(orc):
    cube, idx, anomaly = _scene(40, 48, 14, 3)
    decoy = (0.30 + 0.15 * np.arange(14) / 14).astype(np.float32)
    lib = np.stack([anomaly, decoy])
    s, o, n = orc.moments(cube)
    st, S = orc.build_statistics(s, o, n, lib, 1e-6)
    ace, at, rx, allm = orc.ace(cube, S)
    assert ace.min() >= 0 and ace.max() <= 1
    assert (ace[idx] >= 0.9).all() and (at[idx] == 0).all()
    np.testing.assert_allclose(rx, orc.rx(cube, S), rtol=1e-6)
    cem, ct, _ = orc.cem(cube, S)
    assert ((cem[idx] > 0.8) & (cem[idx] < 1.2)).all()
    # unit gain: w_t . d_t == 1 (tests/test_detector.cpp:227-249)
    gains = (S["cem_weight"] * lib.astype(np.float64)).sum(axis=1)
    np.testing.assert_allclose(gains, 1.0, atol=1e-9)


def test_whitener_reproduces_mahalanobis(orc):
    rng = np.random.default_rng(101)
    X = (0.3 + rng.standard_normal((14, 400)) * 0.05).astype(np.float32)
    s, o, n = orc.moments(X)
    st, S = orc.build_statistics(s, o, n, None, 1e-5)
    cov = o / n - np.outer(s / n, s / n) + 1e-5 * np.eye(14)
    Y = X.astype(np.float64) - (s / n)[:, None]
    want = np.einsum("ip,ij,jp->p", Y, np.linalg.inv(cov), Y)
    got = orc.rx(X, S)
    assert np.max(np.abs(got - want) / np.maximum(1.0, want)) < 1e-4


def test_library_band_mismatch_and_empty(orc):
    X = np.ones((4, 10), np.float32)
    s, o, n = orc.moments(X)
    st, _ = orc.build_statistics(s, o, 0.0, None, 1e-3)
    assert st == orc.STATS_EMPTY


@pytest.mark.parametrize("n", [1, 2, 5, 17])
def test_cholesky_round_trip(orc, n):
    rng = np.random.default_rng(11 + n)
    b = rng.standard_normal((n, n))
    a = b @ b.T + n * np.eye(n)
    l = a.copy()
    assert orc.fp64_lib().orc_cholesky(orc._d(l), n) == 1
    assert np.allclose(np.triu(l, 1), 0)
    assert np.max(np.abs(l @ l.T - a)) < 1e-9
    for bad in (np.zeros((3, 3)), np.array([[1.0, 0], [0, -4.0]]), np.ones((2, 2))):
        m = np.ascontiguousarray(bad, np.float64)
        assert orc.fp64_lib().orc_cholesky(orc._d(m), m.shape[0]) == 0


def test_generator_is_deterministic_and_labelled(orc):
    spec = orc.scene(24, n_targets=3, target_frac=0.05, anomaly_frac=0.02, frame_seed=99)
    a, ta = orc.generate(spec, 16, 20)
    b, tb = orc.generate(spec, 16, 20)
    assert np.array_equal(a, b) and np.array_equal(ta, tb)
    assert a.min() >= 0.0
    labels = set(np.unique(ta).tolist())
    assert 0 in labels and 255 in labels and labels & {1, 2, 3}
    # a sub-range generated on its own equals the same pixels of the whole frame
    part, _ = orc.generate(spec, 2, 20, pixel0=40)
    np.testing.assert_array_equal(part.reshape(24, -1), a.reshape(24, -1)[:, 40:80])
