"""GPU: end-to-end detection-set parity on the benchmark configurations.

Each test runs the product's device chain through the C ABI (generator ->
[moments -> FP64 statistics] -> scorer -> detection list) and compares the
list with the reference's own CPU scorer (oracle/_ref, the reference sources
compiled unmodified) on the same device-generated cube, under the rule stated
in tests/parity.py:

* config 0, plain SAM: 520x696x113, one target in 0.5% of pixels, 0.10 rad,
  sam_best_cpu -> detect_cpu (src/sam_cpu.cpp:48-77,116-138), NMS radius 0
  and 2.  Tolerance 3e-5 rad: the GPU angles are within 2e-5 rad (an FP32
  cosine's rounding grows as 1/sin(angle) near a match) and the reference's
  within 5e-6 rad of the FP64 oracle (both checked here).
* one config-1 frame, SAM+CEM video: 1024x1024x113, 8 targets in 0.2% of
  pixels each; the SAM list (0.10 rad, lower is better) and the CEM list
  (response >= 0.5, higher is better; accumulate_moments_cpu ->
  build_statistics -> cem_best_cpu -> detect_cpu, src/detectors_cpu.cpp:158-187).
  CEM tolerance 1e-4 (the GPU's bar against FP64; the reference is within 1e-5).
* one config-2 frame, RX+ACE precision: 2048x1024x113 with 0.1% anomalies, 8
  ACE targets; the full device chain (tensor-core moments, FP64 factor,
  tensor-core RX/ACE) against the FP64 oracle on EVERY pixel -- RX relative
  <= 1e-4, every ACE map and the ACE best absolute <= 1e-4 -- and the ACE list
  (>= 0.5) against ace_best_cpu -> detect_cpu at radius 0 and 2.

Each test prints its error figures and how many pixels the tolerance band
left out.
"""
import numpy as np
import pytest
import torch

import parity

pytestmark = pytest.mark.gpu

SAM_TOL = 3e-5
SCORE_TOL = 1e-4
LOADING = 1e-6
CAP = 1 << 20


def _host(cube, B, H, W):
    return cube[:, :H * W].float().cpu().numpy().reshape(B, H, W)


def _ref_or_skip(orc):
    if not orc.ref_available():
        pytest.fail("oracle/_ref (the reference's CPU scorer) is missing: run oracle/Makefile")


def _detect(hsi, score, target, H, W, thr, radius, polarity):
    count, out = hsi.detect(score, target, H, W, thr, radius, polarity, CAP)
    torch.cuda.synchronize()
    return parity.gpu_records(hsi, count, out, CAP)


@pytest.mark.parametrize("radius", [0, 2])
def test_config0_sam_list_matches_reference(hsi, orc, radius):
    _ref_or_skip(orc)
    H, W, B = 520, 696, 113
    sc = hsi.scene(B, n_targets=1, target_frac=0.005, library_seed=0x5EED0000, frame_seed=0x5EED0000)
    cube, _ = hsi.generate(sc, H, W)
    targets = hsi.scene_targets(sc)
    P = H * W
    tg = torch.from_numpy(targets).cuda()
    nr = torch.from_numpy(hsi.target_norms(targets)).cuda()
    best = torch.empty(P, device="cuda")
    bt = torch.empty(P, dtype=torch.int32, device="cuda")
    hsi.score_frames([hsi.make_frame(cube, H, W, B, sam_targets=tg, sam_norms=nr, sam_best=best,
                                     sam_best_target=bt, map_stride=P)])
    gpu = _detect(hsi, best, bt, H, W, 0.10, radius, hsi.LOWER_IS_BETTER)

    host = _host(cube, B, H, W)
    rnorms = orc.ref_norms(targets)
    rscore, rwhich = parity.ref_rows_parallel(orc.ref_sam_best, host, targets, rnorms)
    _, ref = orc.ref_detect(rscore, rwhich, H, W, 0.10, radius, False, CAP)
    f64, _ = orc.sam_best(host.reshape(B, P), targets)
    g_err = float(np.abs(best.cpu().numpy() - f64).max())
    r_err = float(np.abs(rscore - f64).max())
    assert g_err <= 2e-5, f"GPU angle error {g_err:.2e} rad"
    assert r_err <= 5e-6, f"reference angle error {r_err:.2e} rad"
    s = parity.compare_lists(gpu, ref, rscore, H, W, 0.10, radius, SAM_TOL)
    assert s["ref"] > 100
    print(f"config 0 r={radius}: {s}, GPU err {g_err:.2e}, reference err {r_err:.2e} rad")


def test_config1_frame_sam_and_cem_lists_match_reference(hsi, orc):
    _ref_or_skip(orc)
    H, W, B, T = 1024, 1024, 113, 8
    sc = hsi.scene(B, n_targets=T, target_frac=0.002, library_seed=0x5EED1000, frame_seed=0x5EED1000)
    cube, _ = hsi.generate(sc, H, W)
    targets = hsi.scene_targets(sc)
    P = H * W
    tg = torch.from_numpy(targets).cuda()
    nr = torch.from_numpy(hsi.target_norms(targets)).cuda()
    # CEM filters from this frame's correlation matrix, all on the device
    gm = hsi.scene_moments(cube, H, W, B)
    cem_w = torch.zeros((T, B), device="cuda")
    _, _, status = hsi.build_statistics(gm, B, tg, loading=LOADING, want64=False, cem_weights=cem_w)
    out = {k: torch.empty(P, device="cuda") for k in ("sb", "cb")}
    out.update({k: torch.empty(P, dtype=torch.int32, device="cuda") for k in ("st", "ct")})
    smaps = torch.empty((T, P), device="cuda")
    cmaps = torch.empty((T, P), device="cuda")
    hsi.score_frames([hsi.make_frame(cube, H, W, B, sam_targets=tg, sam_norms=nr, cem_weights=cem_w,
                                     sam_maps=smaps, sam_best=out["sb"], sam_best_target=out["st"], cem_maps=cmaps,
                                     cem_best=out["cb"], cem_best_target=out["ct"], map_stride=P)])
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    gpu_sam = _detect(hsi, out["sb"], out["st"], H, W, 0.10, 2, hsi.LOWER_IS_BETTER)
    gpu_cem = _detect(hsi, out["cb"], out["ct"], H, W, 0.5, 2, hsi.HIGHER_IS_BETTER)

    host = _host(cube, B, H, W)
    flat = host.reshape(B, P)
    # SAM: reference scorer and list, FP64 per-target maps for the tie margin
    rs, rw = parity.ref_rows_parallel(orc.ref_sam_best, host, targets, orc.ref_norms(targets))
    _, ref_sam = orc.ref_detect(rs, rw, H, W, 0.10, 2, False, CAP)
    sam64 = orc.sam_all(flat, targets)
    s = parity.compare_lists(gpu_sam, ref_sam, rs, H, W, 0.10, 2, SAM_TOL,
                             margin=parity.best_margin(sam64, higher_is_better=False))
    print(f"config 1 SAM: {s}")
    assert s["ref"] > 100

    # CEM: the reference's moments, statistics, scorer and list
    rsum, rout, rn = orc.ref_moments(host)
    ok, msg, RS = orc.ref_build_statistics(rsum, rout, rn, targets, LOADING)
    assert ok, msg
    rc, rcw = parity.ref_rows_parallel(orc.ref_cem_best, host, RS)
    _, ref_cem = orc.ref_detect(rc, rcw, H, W, 0.5, 2, True, CAP)
    # error of both arms against the FP64 oracle
    st, S = orc.build_statistics(*parity.fp64_moments_parallel(orc, flat), targets, LOADING)
    assert st == 0
    c64, _, call64 = orc.cem(flat, S)
    g_err = float(np.abs(cmaps.cpu().numpy() - call64).max())
    r_err = float(np.abs(rc - c64).max())
    assert g_err <= SCORE_TOL, f"GPU CEM error {g_err:.2e}"
    assert r_err <= 1e-5, f"reference CEM error {r_err:.2e}"
    c = parity.compare_lists(gpu_cem, ref_cem, rc, H, W, 0.5, 2, SCORE_TOL,
                             margin=parity.best_margin(call64, higher_is_better=True))
    print(f"config 1 CEM: {c}, GPU err {g_err:.2e}, reference err {r_err:.2e}")
    assert c["ref"] > 100


def test_config2_full_chain_every_pixel_and_ace_list(hsi, orc):
    _ref_or_skip(orc)
    H, W, B, T = 2048, 1024, 113, 8
    sc = hsi.scene(B, n_targets=T, target_frac=0.002, anomaly_frac=0.001, library_seed=0x5EED2000,
                   frame_seed=0x5EED2001)
    cube, _ = hsi.generate(sc, H, W)
    targets = hsi.scene_targets(sc)
    P = H * W
    tg = torch.from_numpy(targets).cuda()
    gm = hsi.scene_moments(cube, H, W, B)
    s64, _, status = hsi.build_statistics(gm, B, tg, loading=LOADING)
    rx = torch.empty(P, device="cuda")
    ace = torch.empty(P, device="cuda")
    at = torch.empty(P, dtype=torch.int32, device="cuda")
    maps = torch.empty((T, P), device="cuda")
    hsi.rx_ace(cube, H, W, B, s64[0], T, rx=rx, ace_best=ace, ace_target=at, ace_maps=maps, simt=False)
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    lists = {r: _detect(hsi, ace, at, H, W, 0.5, r, hsi.HIGHER_IS_BETTER) for r in (0, 2)}

    host = _host(cube, B, H, W)
    flat = host.reshape(B, P)
    st, S = orc.build_statistics(*parity.fp64_moments_parallel(orc, flat), targets, LOADING)
    assert st == 0
    best0, w0, rx0, all0 = parity.fp64_ace_parallel(orc, flat, S)
    rx_g, ace_g, at_g, maps_g = rx.cpu().numpy(), ace.cpu().numpy(), at.cpu().numpy(), maps.cpu().numpy()
    rx_rel = np.abs(rx_g.astype(np.float64) - rx0) / np.maximum(1.0, np.abs(rx0))
    map_err = np.abs(maps_g.astype(np.float64) - all0)
    best_err = np.abs(ace_g.astype(np.float64) - best0)
    print(f"config 2 vs FP64 on {P} px: RX rel max {rx_rel.max():.2e} mean {rx_rel.mean():.2e}; "
          f"ACE maps max {map_err.max(axis=1)} mean {map_err.mean(axis=1)}; best max {best_err.max():.2e}")
    assert rx_rel.max() <= SCORE_TOL
    assert map_err.max() <= SCORE_TOL
    assert best_err.max() <= SCORE_TOL
    for p in np.nonzero(at_g != w0)[0]:
        assert at_g[p] >= 0 and abs(all0[at_g[p], p] - best0[p]) <= SCORE_TOL

    rsum, rout, rn = orc.ref_moments(host)
    ok, msg, RS = orc.ref_build_statistics(rsum, rout, rn, targets, LOADING)
    assert ok, msg
    ra, rw, _ = parity.ref_rows_parallel(orc.ref_ace_best, host, RS)
    r_err = float(np.abs(ra - best0).max())
    assert r_err <= 1e-5, f"reference ACE error {r_err:.2e}"
    margin = parity.best_margin(all0, higher_is_better=True)
    for r in (0, 2):
        _, ref = orc.ref_detect(ra, rw, H, W, 0.5, r, True, CAP)
        s = parity.compare_lists(lists[r], ref, ra, H, W, 0.5, r, SCORE_TOL, margin=margin)
        print(f"config 2 ACE list r={r}: {s}, reference err {r_err:.2e}")
        assert s["ref"] > 100
