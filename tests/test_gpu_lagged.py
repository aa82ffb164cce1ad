"""GPU: the lagged-statistics video runner (include/hsi_lagged.h) against the
oracle run with the lagged statistics.

A stream of frames of one scene model is pushed in order.  Frame k >= 1 must
be scored with frame k-1's statistics and frame 0 with its own, so the oracle
builds the FP64 statistics of the frame before (orc.moments + orc.build_
statistics) and scores frame k with them:
  * SAM maps (statistics-free) within 2e-5 rad of the FP64 oracle (an FP32
    cosine's rounding grows as 1/sin(angle) near a match);
  * CEM maps within 1e-4 of max(1, |response|), RX relative within 1e-4,
    ACE maps within 1e-4;
  * the CEM and ACE lists against the reference's own CPU path fed the same
    lagged statistics (accumulate_moments_cpu + build_statistics of frame k-1,
    then cem_best_cpu / ace_best_cpu and detect_cpu on frame k), under the
    detection-set parity rule of tests/parity.py with tolerance 1e-4 (of
    max(1, |response|) for CEM);
  * the SAM list against sam_best_cpu -> detect_cpu (tolerance 3e-5 rad).
A frame of a different scene in the middle of the stream checks that the
scores really follow the previous frame's statistics (they differ from the
frame's own).
"""
import numpy as np
import pytest
import torch

import parity

pytestmark = pytest.mark.gpu

H, W, B, T = 256, 320, 113, 4
LOADING = 1e-6
TOL = 1e-4


def _frame(hsi, seed, lib_seed):
    sc = hsi.scene(B, n_targets=T, target_frac=0.004, anomaly_frac=0.001, library_seed=lib_seed, frame_seed=seed)
    cube, _ = hsi.generate(sc, H, W)
    return cube


def _arr(hsi, ptr, n, dtype):
    return hsi.device_copy(ptr, n, dtype).cpu().numpy()


def _records(hsi, o, l, cap):
    n = int(_arr(hsi, o.counts, 4, torch.int32)[l])
    k = min(n, cap)
    raw = _arr(hsi, o.detections[l], 4 * k, torch.int32).reshape(k, 4) if k else np.zeros((0, 4), np.int32)
    import oracle
    rec = np.zeros(k, oracle.DETECTION_DTYPE)
    rec["x"], rec["y"], rec["target"] = raw[:, 0], raw[:, 1], raw[:, 2]
    rec["score"] = raw[:, 3].view(np.float32)
    assert n <= cap
    return rec


def test_lagged_stream_matches_oracle_with_previous_statistics(hsi, orc):
    if not orc.ref_available():
        pytest.fail("oracle/_ref is missing: run oracle/Makefile")
    lib_seed = 0x5EED8000
    targets = hsi.scene_targets(hsi.scene(B, n_targets=T, library_seed=lib_seed))
    cap = 1 << 16
    run = hsi.Lagged(H, W, B, targets, loading=LOADING, cem_threshold=0.5, ace_threshold=0.5, nms_radius=2,
                     capacity=cap)
    # frames 0, 1, 3 of one scene; frame 2 of another (another library seed mixes other endmembers)
    cubes = [_frame(hsi, 0x5EED8100 + k, lib_seed if k != 2 else 0x5EED8F00) for k in range(4)]
    hosts = [c[:, :H * W].float().cpu().numpy().reshape(B, H, W) for c in cubes]
    P = H * W
    stream = torch.cuda.current_stream()
    for k, cube in enumerate(cubes):
        run.push(cube, stream)
        torch.cuda.synchronize()
        o = run.outputs()
        assert o.frame == k and o.statistics_frame == max(k - 1, 0)
        assert int(_arr(hsi, o.status, 1, torch.int32)[0]) == 0
        flat = hosts[k].reshape(B, P)
        # FP64 statistics of frame k-1 (of frame 0 for frame 0)
        src = hosts[max(k - 1, 0)].reshape(B, P)
        st, S = orc.build_statistics(*orc.moments(src), targets, LOADING)
        assert st == 0
        rsum, rout, rn = orc.ref_moments(hosts[max(k - 1, 0)])
        ok, msg, RS = orc.ref_build_statistics(rsum, rout, rn, targets, LOADING)
        assert ok, msg

        sam = _arr(hsi, o.sam_maps, T * P, torch.float32).reshape(T, P)
        assert np.abs(sam - orc.sam_all(flat, targets)).max() <= 2e-5
        cem = _arr(hsi, o.cem_maps, T * P, torch.float32).reshape(T, P)
        c64 = orc.cem(flat, S)
        # CEM responses scale with how far the statistics' scene is from the
        # frame's: the bound is 1e-4 of max(1, |response|)
        cerr = (np.abs(cem - c64[2]) / np.maximum(1.0, np.abs(c64[2]))).max()
        assert cerr <= TOL, f"frame {k}: CEM error {cerr:.2e}"
        best0, w0, rx0, all0 = orc.ace(flat, S)
        rx = _arr(hsi, o.rx, P, torch.float32)
        assert (np.abs(rx - rx0) / np.maximum(1.0, np.abs(rx0))).max() <= TOL
        ace = _arr(hsi, o.ace_maps, T * P, torch.float32).reshape(T, P)
        assert np.abs(ace - all0).max() <= TOL

        # lists against the reference CPU path with the same lagged statistics
        rc, rcw = orc.ref_cem_best(hosts[k], RS)
        _, ref_cem = orc.ref_detect(rc, rcw, H, W, 0.5, 2, True, cap)
        cs = parity.compare_lists(_records(hsi, o, 1, cap), ref_cem, rc, H, W, 0.5, 2, TOL,
                                  margin=parity.best_margin(c64[2], True), rel=True)
        ra, rw, _ = orc.ref_ace_best(hosts[k], RS)
        _, ref_ace = orc.ref_detect(ra, rw, H, W, 0.5, 2, True, cap)
        a = parity.compare_lists(_records(hsi, o, 2, cap), ref_ace, ra, H, W, 0.5, 2, TOL,
                                 margin=parity.best_margin(all0, True))
        rs, rsw = orc.ref_sam_best(hosts[k], targets, orc.ref_norms(targets))
        _, ref_sam = orc.ref_detect(rs, rsw, H, W, 0.10, 2, False, cap)
        m = parity.compare_lists(_records(hsi, o, 0, cap), ref_sam, rs, H, W, 0.10, 2, 3e-5,
                                 margin=parity.best_margin(orc.sam_all(flat, targets), False))
        print(f"lagged frame {k}: CEM {cs}, ACE {a}, SAM {m}")
        if k == 3:
            # frame 3 follows the other scene's frame: its scores use frame 2's
            # statistics and differ clearly from scores with its own
            _, S3 = orc.build_statistics(*orc.moments(flat), targets, LOADING)
            own = orc.ace(flat, S3)[3]
            assert np.abs(own - ace).max() > 100 * TOL
