"""hsi_detect, the reference's command-line consumer (src/main.cpp) on this library.

CPU: the binary builds, --help lists the reference's flags and the added ones,
and usage errors exit 2 with their message before any device call.
GPU: each detector runs end to end on small synthetic frames and reports.
"""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "hsi-detectors-cuda_b200")
CLI = os.path.join(PKG, "build", "hsi_detect")


def _build():
    subprocess.run(["make", "-s", "-j8", "-C", PKG, "all"], check=True, capture_output=True, text=True)


def _run(*args, timeout=120):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=timeout)


def test_help_lists_the_reference_flags_and_the_added_ones():
    _build()
    r = _run("--help")
    assert r.returncode == 0
    for flag in ["--source=", "--envi=", "--resident=", "--width=", "--height=", "--bands=", "--targets=", "--noise=", "--library=",
                 "--threshold=", "--nms=", "--max-detections=", "--variant=", "--memory=", "--streams=",
                 "--frames=", "--warmup=", "--prefill", "--csv=", "--print-detections=", "--dump-score=",
                 "--quiet", "--detector=sam|cem|rx|ace", "--batch", "--repeat=", "--pfa=", "--loading=",
                 "--lagged"]:
        assert flag in r.stdout, flag


@pytest.mark.parametrize("args, message", [
    (["--source=envi"], "--source=envi needs --envi=<header>[,<header>...]"),
    (["--source=hot"], "not built in this library"),
    (["--source=tape"], "unknown --source=tape"),
    (["--detector=mahalanobis"], "--detector must be sam, cem, rx or ace"),
    (["--variant=fast"], "--variant must be baseline, optimized or half"),
    (["--memory=pinned"], "--memory must be copy or zerocopy"),
    (["--frames=ten"], "--frames must be an integer"),
    (["--bands=300"], "--bands must be an integer in [1, 256]"),
    (["--nms=-1"], "--nms must be an integer"),
    (["--pfa=1.5"], "--pfa must lie in (0, 1)"),
    (["--batch", "--detector=cem"], "--batch lists SAM, ACE and RX detections"),
    (["--batch", "--frames=65"], "--batch takes at most 64 frames"),
    (["--lagged"], "--lagged needs --detector=cem, rx or ace"),
    (["--lagged", "--detector=ace", "--batch"], "--lagged and --batch are separate modes"),
    (["--lagged", "--detector=rx", "--threshold=50"], "--lagged sets the RX threshold from --pfa"),
])
def test_usage_errors_exit_2_before_any_device_call(args, message):
    _build()
    r = _run(*args)
    assert r.returncode == 2, r.stdout + r.stderr
    assert message in r.stderr, r.stderr


def test_reference_variant_names_are_accepted():
    """"optimized" (the reference CLI's default), "opt", "fp16", "zero-copy" parse; the
    run then stops at the missing library file, before any device call."""
    _build()
    for extra in (["--variant=optimized"], ["--variant=opt"], ["--variant=fp16"], ["--memory=zero-copy"]):
        r = _run("--library=/nonexistent/lib.csv", *extra)
        assert r.returncode == 1, r.stderr
        assert "cannot open spectral library" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("detector", ["sam", "cem", "rx", "ace"])
def test_each_detector_runs_end_to_end(detector):
    _build()
    r = _run(f"--detector={detector}", "--width=256", "--height=192", "--bands=64", "--frames=6", "--warmup=2",
             "--print-detections=2", timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "frames 6 in" in r.stdout and "detections" in r.stdout, r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("detector", ["cem", "rx", "ace"])
def test_lagged_mode_runs(detector):
    _build()
    r = _run("--lagged", f"--detector={detector}", "--width=256", "--height=192", "--bands=64", "--frames=6",
             "--warmup=2", "--print-detections=2", timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "lagged: frame k scored with frame k-1's statistics" in r.stdout and "frames 6 in" in r.stdout, r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("detector", ["sam", "ace", "rx"])
def test_batch_mode_runs(detector):
    _build()
    r = _run("--batch", f"--detector={detector}", "--width=256", "--height=192", "--bands=64", "--frames=4",
             "--warmup=1", "--repeat=3", "--print-detections=2", timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "batch of 4 frames" in r.stdout, r.stdout


def _envi_cube(tmp_path, name, H, W, B, seed):
    import numpy as np
    rng = np.random.default_rng(seed)
    cube = rng.uniform(0.05, 1.0, (H, W, B)).astype("<f4")  # BIP order
    (tmp_path / name).write_bytes(cube.tobytes())
    (tmp_path / (name + ".hdr")).write_text(
        f"ENVI\nsamples = {W}\nlines = {H}\nbands = {B}\ndata type = 4\ninterleave = bip\nbyte order = 0\n")
    return str(tmp_path / (name + ".hdr"))


def test_envi_source_errors_before_any_device_call(tmp_path):
    """An ENVI replay without --library stops at the missing library (exit 2), an unreadable
    header at the reader (exit 1), both before the device is used."""
    _build()
    hdr = _envi_cube(tmp_path, "scene", 4, 6, 5, 1)
    r = _run("--source=envi", f"--envi={hdr}")
    assert r.returncode == 2 and "no target spectra: pass --library=<csv>" in r.stderr, r.stderr
    r = _run("--source=envi", f"--envi={tmp_path / 'missing.hdr'}", "--library=/nonexistent.csv")
    assert r.returncode == 1 and "cannot open spectral library" in r.stderr, r.stderr
    lib = tmp_path / "lib.csv"
    lib.write_text("a,0.1,0.2,0.3,0.4,0.5\n")
    r = _run("--source=envi", f"--envi={tmp_path / 'missing.hdr'}", f"--library={lib}")
    assert r.returncode == 1 and "cannot open ENVI header" in r.stderr, r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("detector", ["sam", "ace"])
def test_envi_replay_runs_end_to_end(tmp_path, detector):
    _build()
    a = _envi_cube(tmp_path, "a", 64, 96, 24, 2)
    b = _envi_cube(tmp_path, "b", 64, 96, 24, 3)
    lib = tmp_path / "lib.csv"
    lib.write_text("t0," + ",".join(f"{0.2 + 0.01 * i:.3f}" for i in range(24)) + "\n"
                   + "t1," + ",".join(f"{0.9 - 0.02 * i:.3f}" for i in range(24)) + "\n")
    r = _run("--source=envi", f"--envi={a},{b}", f"--library={lib}", f"--detector={detector}", "--frames=4",
             "--warmup=1", timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "envi-replay(2 cubes, 64x96x24)" in r.stdout and "frames 4 in" in r.stdout, r.stdout
