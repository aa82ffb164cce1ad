"""Generate the golden fixtures in this folder from the reference's own CPU code.

Run in a checkout that has the reference tree (it builds oracle/_ref from the
reference sources with oracle/Makefile, then calls it through ctypes):

    python tests/golden/make_golden.py

Every output array here was produced by the reference's unmodified functions
(src/sam_cpu.cpp, src/detectors_cpu.cpp, src/detector.cpp, src/linalg.cpp,
src/hot_loader.cpp, src/frame_source.cpp).  Inputs are either generated by the
scene model in csrc/synth.h (seeded) or are the small hand-built cases the
reference's own tests use (tests/test_sam.cpp, tests/test_detector.cpp,
tests/test_linalg.cpp), rebuilt here from their descriptions.

The fixtures pin the project's FP64 oracle (oracle/hsi_oracle.c) and are also
replayed against the GPU path by the -m gpu tests.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

import oracle as O  # noqa: E402


def correlated_scene(h, w, bands, seed, anomalies=True):
    """A smooth background with two shared factors plus noise, and three planted
    inverted-ramp anomalies - the kind of scene the reference's detector tests
    build (tests/test_detectors.cpp:24-60)."""
    rng = np.random.default_rng(seed)
    P = h * w
    t = np.arange(bands, dtype=np.float32) / np.float32(bands)
    a = (rng.standard_normal(P) * 0.05).astype(np.float32)
    b = (rng.standard_normal(P) * 0.03).astype(np.float32)
    cube = (0.30 + 0.15 * t[:, None] + a[None, :] * (t * (1 - t))[:, None]
            + b[None, :] * np.sin(4 * t)[:, None]
            + rng.standard_normal((bands, P)) * 0.01).astype(np.float32)
    anomaly = (0.75 - 0.55 * t).astype(np.float32)
    idx = np.array([P // 7, P // 3, (2 * P) // 3]) if anomalies else np.zeros(0, np.int64)
    for p in idx:
        cube[:, p] = anomaly + (rng.standard_normal(bands) * 0.01).astype(np.float32)
    return cube.reshape(bands, h, w), idx, anomaly


def random_spd(n, rng):
    b = rng.standard_normal((n, n))
    return b @ b.T + n * np.eye(n)


def main():
    O.build()
    assert O.ref_available(), "the reference build oracle/_ref/libhsi_ref.so is missing"
    g = {}

    # --- SAM + detection on a generated scene (config-0 model, 3 targets) ---
    spec = O.scene(16, n_targets=3, target_frac=0.02, library_seed=0x5EED0001, frame_seed=0x5EED0101)
    cube, truth = O.generate(spec, 24, 32)
    _, targets, _ = O.scene_spectra(spec.library_seed, 16, 6, 3)
    norms = O.ref_norms(targets)
    score, which = O.ref_sam_best(cube, targets, norms)
    g.update(sam_cube=cube, sam_targets=targets, sam_norms=norms, sam_best_score=score,
             sam_best_target=which, sam_all=O.ref_sam_all(cube, targets, norms))
    thr = float(np.quantile(score, 0.10))
    g["sam_threshold"] = np.float32(thr)
    for r in (0, 1, 2, 3):
        n, d = O.ref_detect(score, which, 24, 32, thr, r, False)
        g[f"sam_detect_r{r}"] = d
    # the same map read as higher-is-better
    thr_hi = float(np.quantile(score, 0.90))
    g["sam_threshold_hi"] = np.float32(thr_hi)
    for r in (0, 2):
        n, d = O.ref_detect(score, which, 24, 32, thr_hi, r, True)
        g[f"sam_detect_hi_r{r}"] = d

    # --- the reference's own hand-built SAM / NMS cases (tests/test_sam.cpp) ---
    # identical spectrum -> 0 angle
    t8 = np.array([[0.1, 0.4, 0.9, 0.3, 0.2, 0.7, 0.5, 0.6]], np.float32)
    s, w = O.ref_sam_best(t8.T.reshape(8, 1, 1), t8, O.ref_norms(t8))
    g.update(case_identical_cube=t8.T.reshape(8, 1, 1), case_identical_targets=t8,
             case_identical_score=s, case_identical_target=w)
    # orthogonal + all-zero pixel -> pi/2
    cz = np.zeros((4, 1, 2), np.float32)
    cz[:, 0, 0] = [0, 1, 0, 1]
    tz = np.array([[1, 0, 1, 0]], np.float32)
    s, w = O.ref_sam_best(cz, tz, O.ref_norms(tz))
    g.update(case_zero_cube=cz, case_zero_targets=tz, case_zero_score=s, case_zero_target=w)
    # best match among three
    pix = np.array([0.1, 0.2, 0.3, 0.4, 0.5, 0.6], np.float32).reshape(6, 1, 1)
    t3 = np.array([[1, 0, 0, 0, 0, 0], [0.2, 0.4, 0.6, 0.8, 1.0, 1.2], [0.6, 0.5, 0.4, 0.3, 0.2, 0.1]],
                  np.float32)
    s, w = O.ref_sam_best(pix, t3, O.ref_norms(t3))
    g.update(case_best_cube=pix, case_best_targets=t3, case_best_score=s, case_best_target=w,
             case_best_all=O.ref_sam_all(pix, t3, O.ref_norms(t3)))
    # NMS: one pixel per blob, plateau tie-break, polarity
    blob = np.ones((9, 9), np.float32)
    blob[3:6, 3:6] = 0.05
    blob[4, 4] = 0.01
    g["case_blob_score"] = blob
    for r in (0, 2):
        g[f"case_blob_detect_r{r}"] = O.ref_detect(blob, np.zeros(81, np.int32), 9, 9, 0.1, r, False)[1]
    plateau = np.ones((5, 5), np.float32)
    plateau[1:3, 1:3] = 0.02
    g["case_plateau_score"] = plateau
    g["case_plateau_detect"] = O.ref_detect(plateau, np.zeros(25, np.int32), 5, 5, 0.1, 2, False)[1]
    pol = np.full((7, 7), 0.5, np.float32)
    pol[2, 2] = 0.01
    pol[5, 5] = 0.99
    g["case_polarity_score"] = pol
    g["case_polarity_low"] = O.ref_detect(pol, np.zeros(49, np.int32), 7, 7, 0.1, 1, False)[1]
    g["case_polarity_high"] = O.ref_detect(pol, np.zeros(49, np.int32), 7, 7, 0.9, 1, True)[1]
    ext = np.full((9, 9), 0.5, np.float32)
    ext[3:6, 3:6] = 0.8
    ext[3, 3] = 0.6
    ext[5, 5] = 0.95
    g["case_extremum_score"] = ext
    g["case_extremum_high"] = O.ref_detect(ext, np.zeros(81, np.int32), 9, 9, 0.55, 3, True)[1]

    # --- moments, statistics, RX / ACE / CEM (tests/test_detectors.cpp) ---
    sc, anomalies, anomaly = correlated_scene(20, 24, 12, seed=3)
    decoy = (0.30 + 0.15 * np.arange(12, dtype=np.float32) / 12).astype(np.float32)
    lib = np.stack([anomaly, decoy]).astype(np.float32)
    s1, m2, cnt = O.ref_moments(sc)
    ok, msg, st = O.ref_build_statistics(s1, m2, cnt, lib, 1e-6)
    assert ok, msg
    ace_s, ace_t, ace_rx = O.ref_ace_best(sc, st)
    cem_s, cem_t = O.ref_cem_best(sc, st)
    g.update(stats_cube=sc, stats_anomalies=anomalies, stats_library=lib, stats_loading=np.float64(1e-6),
             stats_sum=s1, stats_outer=m2, stats_count=np.float64(cnt),
             stats_mean=st["mean"], stats_whitener=st["whitener"], stats_target_white=st["target_white"],
             stats_target_norm2=st["target_norm2"], stats_cem_weight=st["cem_weight"],
             stats_rx=O.ref_rx(sc, st), stats_ace=ace_s, stats_ace_target=ace_t, stats_ace_rx=ace_rx,
             stats_cem=cem_s, stats_cem_target=cem_t)

    # generated config-2-style scene at 113 bands, 8 targets + anomalies
    spec2 = O.scene(113, n_targets=8, target_frac=0.01, anomaly_frac=0.01,
                    library_seed=0x5EED2000, frame_seed=0x5EED2001)
    c2, truth2 = O.generate(spec2, 16, 24)
    _, lib2, _ = O.scene_spectra(spec2.library_seed, 113, 6, 8)
    s1, m2, cnt = O.ref_moments(c2)
    ok, msg, st2 = O.ref_build_statistics(s1, m2, cnt, lib2, 1e-5)
    assert ok, msg
    a2, at2, ar2 = O.ref_ace_best(c2, st2)
    cs2, ct2 = O.ref_cem_best(c2, st2)
    g.update(b113_cube=c2, b113_library=lib2, b113_loading=np.float64(1e-5), b113_sum=s1, b113_outer=m2,
             b113_count=np.float64(cnt), b113_mean=st2["mean"], b113_whitener=st2["whitener"],
             b113_target_white=st2["target_white"], b113_target_norm2=st2["target_norm2"],
             b113_cem_weight=st2["cem_weight"], b113_ace=a2, b113_ace_target=at2, b113_rx=ar2,
             b113_cem=cs2, b113_cem_target=ct2)

    # singular covariance (tests/test_detector.cpp:251-275)
    rng = np.random.default_rng(5)
    shared = rng.normal(0.5, 0.1, 100).astype(np.float32)
    other = rng.normal(0.5, 0.1, 100).astype(np.float32)
    sing = np.stack([shared, shared, other, other]).reshape(4, 10, 10)
    s1, m2, cnt = O.ref_moments(sing)
    ok0, msg0, _ = O.ref_build_statistics(s1, m2, cnt, None, 0.0)
    ok1, _, _ = O.ref_build_statistics(s1, m2, cnt, None, 1e-3)
    g.update(singular_cube=sing, singular_ok_unloaded=np.int32(ok0), singular_ok_loaded=np.int32(ok1),
             singular_message=np.array(msg0))

    # --- linear algebra (tests/test_linalg.cpp) ---
    rng = np.random.default_rng(11)
    a = random_spd(17, rng)
    l = np.ascontiguousarray(a.copy())
    O.ref_lib().ref_cholesky(O._d(l), 17)
    inv = np.zeros((17, 17))
    O.ref_lib().ref_triangular_inverse_lower(O._d(l), 17, O._d(inv))
    bvec = rng.standard_normal(17)
    x = np.zeros(17)
    O.ref_lib().ref_cholesky_solve(O._d(l), 17, O._d(bvec), O._d(x))
    g.update(linalg_a=a, linalg_l=l, linalg_inv=inv, linalg_b=bvec, linalg_x=x)
    # shifted moments
    xs = rng.normal(0.4, 0.05, (300, 5)).astype(np.float32)
    ref = np.full(5, 0.41)
    d = xs.astype(np.float64) - ref
    s1 = d.sum(0)
    s2 = np.tril(d.T @ d)
    msum = np.zeros(5)
    mout = np.zeros((5, 5))
    O.ref_lib().ref_moments_from_shifted(O._d(s1), O._d(np.ascontiguousarray(s2)), 300.0, O._d(ref), 5,
                                         O._d(msum), O._d(mout))
    g.update(shift_s1=s1, shift_s2=s2, shift_ref=ref, shift_sum=msum, shift_outer=mout)

    # --- chi-squared thresholds ---
    table = [(2, 0.5), (2, 0.1), (2, 1e-3), (2, 1e-6), (12, 1e-3), (50, 1e-6), (50, 1e-2), (100, 0.5),
             (113, 1e-3), (224, 1e-3), (16, 1e-3)]
    g["chi2_cases"] = np.array(table, np.float64)
    g["chi2_thresholds"] = np.array([O.ref_rx_threshold(b, r) for b, r in table], np.float64)

    # --- demosaic (src/hot_loader.cpp:144-182) ---
    raw = (np.arange(16 * 24, dtype=np.float32) / 384.0).reshape(16, 24)
    order = np.array([(5 * i + 3) % 16 for i in range(16)], np.int32)
    g.update(demosaic_raw=raw, demosaic_order=order, demosaic_16=O.ref_demosaic(raw, 4, 16),
             demosaic_16_ordered=O.ref_demosaic(raw, 4, 16, order), demosaic_15=O.ref_demosaic(raw, 4, 15))

    # --- the reference's own synthetic video frame, for the end-to-end check
    #     (tests/test_sources.cpp:83-144) ---
    cube_s, truth_s, lib_s = O.ref_synthetic_frame(48, 64, 24, num_targets=3, target_radius=5, seed=4242)
    g.update(source_cube=cube_s, source_truth=truth_s, source_library=lib_s)

    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **g)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB, {len(g)} arrays)")


if __name__ == "__main__":
    main()
