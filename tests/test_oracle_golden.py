"""Pin the FP64 oracle (oracle/hsi_oracle.c) against the reference's own outputs.

The fixtures in tests/golden/golden.npz were produced by the reference's
unmodified CPU code (tests/golden/make_golden.py).  Integer and index results
must match exactly; floating-point results within the stated tolerances (the
reference narrows its statistics to float, the oracle keeps them in double).
"""
import numpy as np
import pytest


def _det_tuples(d):
    return [(int(r["x"]), int(r["y"]), int(r["target"]), float(r["score"])) for r in d]


def test_sam_best_matches_reference(golden, orc):
    cube, tg = golden["sam_cube"], golden["sam_targets"]
    assert np.array_equal(orc.target_norms(tg), golden["sam_norms"])
    score, which = orc.sam_best(cube, tg)
    assert np.array_equal(which, golden["sam_best_target"])
    assert np.max(np.abs(score - golden["sam_best_score"])) == 0.0  # same double arithmetic
    allm = orc.sam_all(cube, tg)
    assert np.max(np.abs(allm - golden["sam_all"])) == 0.0


@pytest.mark.parametrize("radius", [0, 1, 2, 3])
def test_detect_matches_reference_bit_exact(golden, orc, radius):
    score, which = golden["sam_best_score"], golden["sam_best_target"]
    n, d = orc.detect(score, which, 24, 32, float(golden["sam_threshold"]), radius, False)
    want = golden[f"sam_detect_r{radius}"]
    assert n == len(want)
    assert _det_tuples(d) == _det_tuples(want)


@pytest.mark.parametrize("radius", [0, 2])
def test_detect_higher_is_better_matches_reference(golden, orc, radius):
    score, which = golden["sam_best_score"], golden["sam_best_target"]
    n, d = orc.detect(score, which, 24, 32, float(golden["sam_threshold_hi"]), radius, True)
    assert _det_tuples(d) == _det_tuples(golden[f"sam_detect_hi_r{radius}"])


def test_reference_hand_built_sam_cases(golden, orc):
    s, w = orc.sam_best(golden["case_identical_cube"], golden["case_identical_targets"])
    assert abs(s[0] - golden["case_identical_score"][0]) < 1e-6 and abs(s[0]) < 1e-5 and w[0] == 0
    s, w = orc.sam_best(golden["case_zero_cube"], golden["case_zero_targets"])
    np.testing.assert_array_equal(s, golden["case_zero_score"])
    assert not np.isnan(s).any()
    s, w = orc.sam_best(golden["case_best_cube"], golden["case_best_targets"])
    assert w[0] == golden["case_best_target"][0] == 1
    np.testing.assert_allclose(orc.sam_all(golden["case_best_cube"], golden["case_best_targets"]),
                               golden["case_best_all"], atol=0)


def test_reference_hand_built_nms_cases(golden, orc):
    z = lambda n: np.zeros(n, np.int32)  # noqa: E731
    for r in (0, 2):
        n, d = orc.detect(golden["case_blob_score"], z(81), 9, 9, 0.1, r, False)
        assert _det_tuples(d) == _det_tuples(golden[f"case_blob_detect_r{r}"])
    assert len(golden["case_blob_detect_r0"]) == 9 and len(golden["case_blob_detect_r2"]) == 1
    n, d = orc.detect(golden["case_plateau_score"], z(25), 5, 5, 0.1, 2, False)
    assert _det_tuples(d) == _det_tuples(golden["case_plateau_detect"]) == [(1, 1, 0, pytest.approx(0.02))]
    n, d = orc.detect(golden["case_polarity_score"], z(49), 7, 7, 0.1, 1, False)
    assert _det_tuples(d) == _det_tuples(golden["case_polarity_low"])
    n, d = orc.detect(golden["case_polarity_score"], z(49), 7, 7, 0.9, 1, True)
    assert _det_tuples(d) == _det_tuples(golden["case_polarity_high"])
    n, d = orc.detect(golden["case_extremum_score"], z(81), 9, 9, 0.55, 3, True)
    assert _det_tuples(d) == _det_tuples(golden["case_extremum_high"])


def test_moments_match_reference(golden, orc):
    s, o, n = orc.moments(golden["stats_cube"])
    assert n == golden["stats_count"]
    np.testing.assert_allclose(s, golden["stats_sum"], rtol=1e-13)
    np.testing.assert_allclose(np.tril(o), np.tril(golden["stats_outer"]), rtol=1e-13)


@pytest.mark.parametrize("prefix", ["stats", "b113"])
def test_statistics_and_detectors_match_reference(golden, orc, prefix):
    g = lambda k: golden[f"{prefix}_{k}"]  # noqa: E731
    cube = g("cube")
    st, S = orc.build_statistics(g("sum"), g("outer"), float(g("count")), g("library"), float(g("loading")))
    assert st == orc.STATS_OK
    # the reference narrows to float: agreement is at float resolution
    rel = lambda a, b: np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30)  # noqa: E731
    assert rel(S["mean"], g("mean")) < 1e-6
    assert rel(S["whitener"], g("whitener")) < 1e-5
    assert rel(S["target_white"], g("target_white")) < 1e-5
    assert rel(S["target_norm2"], g("target_norm2")) < 1e-5
    assert rel(S["cem_weight"], g("cem_weight")) < 1e-5
    assert np.allclose(np.triu(S["whitener"], 1), 0.0)
    rx = orc.rx(cube, S)
    want_rx = g("ace_rx") if prefix == "stats" else g("rx")
    assert np.max(np.abs(rx - want_rx) / np.maximum(1.0, np.abs(want_rx))) < 1e-4
    ace, at, arx, _ = orc.ace(cube, S)
    assert np.max(np.abs(ace - g("ace"))) < 1e-4
    confident = np.abs(ace - g("ace")) < 1e-6
    assert np.array_equal(at[confident & (g("ace") > 0.05)], g("ace_target")[confident & (g("ace") > 0.05)])
    cem, ct, _ = orc.cem(cube, S)
    assert np.max(np.abs(cem - g("cem"))) < 1e-4
    assert np.mean(ct == g("cem_target")) > 0.99


def test_singular_covariance_reports_loading(golden, orc):
    s, o, n = orc.moments(golden["singular_cube"])
    st0, _ = orc.build_statistics(s, o, n, None, 0.0)
    st1, _ = orc.build_statistics(s, o, n, None, 1e-3)
    assert (st0 == orc.STATS_OK) == bool(golden["singular_ok_unloaded"])
    assert st0 == orc.STATS_COVARIANCE_NOT_PD
    assert "loading" in str(golden["singular_message"])
    assert (st1 == orc.STATS_OK) == bool(golden["singular_ok_loaded"])


def test_linalg_matches_reference(golden, orc):
    a = golden["linalg_a"].copy()
    L = orc.fp64_lib()
    assert L.orc_cholesky(orc._d(a), 17) == 1
    np.testing.assert_allclose(a, golden["linalg_l"], rtol=0, atol=1e-12)
    inv = np.zeros((17, 17))
    L.orc_triangular_inverse_lower(orc._d(golden["linalg_l"].copy()), 17, orc._d(inv))
    np.testing.assert_allclose(inv, golden["linalg_inv"], atol=1e-14)
    x = np.zeros(17)
    L.orc_cholesky_solve(orc._d(golden["linalg_l"].copy()), 17, orc._d(golden["linalg_b"].copy()), orc._d(x))
    np.testing.assert_allclose(x, golden["linalg_x"], atol=1e-13)
    s = np.zeros(5)
    o = np.zeros((5, 5))
    L.orc_moments_from_shifted(orc._d(golden["shift_s1"].copy()), orc._d(golden["shift_s2"].copy()), 300.0,
                               orc._d(golden["shift_ref"].copy()), 5, orc._d(s), orc._d(o))
    np.testing.assert_allclose(s, golden["shift_sum"], rtol=1e-15)
    np.testing.assert_allclose(np.tril(o), np.tril(golden["shift_outer"]), rtol=1e-14)


def test_chi_squared_thresholds_match_reference(golden, orc):
    for (b, r), want in zip(golden["chi2_cases"], golden["chi2_thresholds"]):
        got = orc.rx_threshold(int(b), float(r))
        assert abs(got - want) <= 1e-9 * max(1.0, want)
    # closed form at 2 degrees of freedom (reference tests/test_detectors.cpp:214-228)
    for r in (0.5, 0.1, 1e-3, 1e-6):
        assert abs(orc.rx_threshold(2, r) + 2 * np.log(r)) < 1e-6 * max(1.0, -2 * np.log(r))
    assert np.isnan(orc.rx_threshold(0, 0.1)) and np.isnan(orc.rx_threshold(10, 1.5))


def test_demosaic_matches_reference(golden, orc):
    raw = golden["demosaic_raw"]
    np.testing.assert_array_equal(orc.demosaic(raw, 4, 16), golden["demosaic_16"])
    np.testing.assert_array_equal(orc.demosaic(raw, 4, 16, golden["demosaic_order"]), golden["demosaic_16_ordered"])
    np.testing.assert_array_equal(orc.demosaic(raw, 4, 15), golden["demosaic_15"])
    assert orc.demosaic(raw, 4, 17) is None


def test_reference_source_frame_end_to_end(golden, orc):
    """tests/test_sources.cpp:83-144 on the reference's own generated frame."""
    cube, truth, lib = golden["source_cube"], golden["source_truth"], golden["source_library"]
    score, which = orc.sam_best(cube, lib)
    n, found = orc.detect(score, which, 48, 64, 0.05, 4, False)
    assert n > 0
    for d in found:
        t = truth[d["y"], d["x"]]
        assert t != 0 and t - 1 == d["target"]
    assert len(set(int(d["target"]) for d in found)) == lib.shape[0]
    assert score[truth.reshape(-1) == 0].min() > 0.05
