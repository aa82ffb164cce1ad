"""GPU: hsi_detect's detections against the reference's own CPU path.

The reference's consumer is its command-line tool (src/main.cpp:125-292).
This runs ours end to end -- ENVI replay of two cubes written here, the CSV
target library, upload, statistics, scoring, detection, the printed list of
the last frame -- and compares the printed list with the reference's CPU
scorer and detect_cpu on the same cube (oracle/_ref), under the
detection-set parity rule of tests/parity.py:
  * sam: sam_best_cpu -> detect_cpu, 0.25 rad (--threshold), lower is better;
  * cem / ace: accumulate_moments_cpu + build_statistics of the frame, then
    cem_best_cpu / ace_best_cpu -> detect_cpu at 0.5, higher is better;
  * rx: ace_best_cpu's RX map -> detect_cpu at the reference's chi-square
    threshold for --pfa;
  * --lagged cem / ace: the statistics of the frame before (the first cube),
    the scores of the last frame (the second cube).
Printed scores carry 4 decimals, so scores are compared within 2e-4
(RX: 1e-4 of the value, plus the print's 5e-5).
"""
import os
import re
import subprocess

import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "hsi-detectors-cuda_b200", "build", "hsi_detect")
H, W, B, T = 96, 128, 32, 3
LOADING = 1e-6
PFA = 1e-3
LINE = re.compile(r"\(\s*(-?\d+),\s*(-?\d+)\) target (-?\d+)\s+\w+ (-?[\d.]+)")


def _write_envi(tmp_path, name, cube):
    bip = np.ascontiguousarray(cube.transpose(1, 2, 0), "<f4")  # (H, W, B)
    (tmp_path / name).write_bytes(bip.tobytes())
    (tmp_path / (name + ".hdr")).write_text(
        f"ENVI\nsamples = {W}\nlines = {H}\nbands = {B}\ndata type = 4\ninterleave = bip\nbyte order = 0\n")
    return str(tmp_path / (name + ".hdr"))


def _scene(orc):
    lib_seed = 0x5EED9000
    cubes = []
    for k in range(2):
        sc = orc.scene(B, n_targets=T, target_frac=0.01, anomaly_frac=0.002, library_seed=lib_seed,
                       frame_seed=0x5EED9100 + k)
        cubes.append(orc.generate(sc, H, W)[0])
    targets = orc.scene_spectra(lib_seed, B, n_targets=T)[1].astype(np.float32)
    return cubes, targets


def _printed(stdout):
    tail = stdout.split("detections:", 1)[1]
    rows = [m.groups() for m in LINE.finditer(tail)]
    import oracle
    rec = np.zeros(len(rows), oracle.DETECTION_DTYPE)
    for i, (x, y, t, s) in enumerate(rows):
        rec[i] = (int(x), int(y), int(t), float(s))
    return rec


@pytest.mark.parametrize("detector, lagged", [("sam", False), ("cem", False), ("ace", False), ("rx", False),
                                              ("cem", True), ("ace", True), ("rx", True)])
def test_cli_lists_match_reference(tmp_path, orc, detector, lagged):
    if not orc.ref_available():
        pytest.fail("oracle/_ref is missing: run oracle/Makefile")
    cubes, targets = _scene(orc)
    hdrs = [_write_envi(tmp_path, f"f{k}", c) for k, c in enumerate(cubes)]
    lib = tmp_path / "lib.csv"
    lib.write_text("".join(f"t{t}," + ",".join(repr(float(v)) for v in targets[t]) + "\n" for t in range(T)))
    cap = 100000
    args = [CLI, "--source=envi", f"--envi={hdrs[0]},{hdrs[1]}", f"--library={lib}", f"--detector={detector}",
            "--frames=2", "--warmup=0", "--nms=2", f"--print-detections={cap}", f"--max-detections={cap}",
            f"--pfa={PFA}", f"--loading={LOADING}"]
    if lagged:
        args.append("--lagged")
    if detector == "sam":
        args.append("--threshold=0.25")
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = _printed(r.stdout)

    last = cubes[1]
    flat = last.reshape(B, H * W)
    stats_src = cubes[0] if lagged else cubes[1]
    rel, margin = False, None
    if detector == "sam":
        score, which = orc.ref_sam_best(last, targets, orc.ref_norms(targets))
        thr, higher, tol = 0.25, False, 2e-4
        margin = parity.best_margin(orc.sam_all(flat, targets), False)
    else:
        ok, msg, RS = orc.ref_build_statistics(*orc.ref_moments(stats_src), targets, LOADING)
        assert ok, msg
        st, S = orc.build_statistics(*orc.moments(stats_src.reshape(B, H * W)), targets, LOADING)
        assert st == 0
        if detector == "cem":
            score, which = orc.ref_cem_best(last, RS)
            thr, higher, tol, rel = 0.5, True, 2e-4, True
            margin = parity.best_margin(orc.cem(flat, S)[2], True)
        else:
            ace, at, rxm = orc.ref_ace_best(last, RS)
            if detector == "ace":
                score, which, thr, higher, tol = ace, at, 0.5, True, 2e-4
                margin = parity.best_margin(orc.ace(flat, S)[3], True)
            else:
                score, which, higher, tol, rel = rxm, None, True, 1.5e-4, True
                thr = float(np.float32(orc.ref_rx_threshold(B, PFA)))
    n, ref = orc.ref_detect(score, which, H, W, thr, 2, higher, cap)
    assert n == len(ref) and len(got) > 0
    s = parity.compare_lists(got, ref, score, H, W, thr, 2, tol, margin=margin, rel=rel)
    print(f"hsi_detect {detector}{' --lagged' if lagged else ''}: {s}")
