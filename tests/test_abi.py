"""The C-ABI libraries load and export every entry point include/*.h declares:
include/hsi_b200.h from libhsi_b200.so (kernels), include/hsi_batch.h and
include/hsi_lagged.h from libhsi_cxx.so (the batch and lagged-statistics
runners, host C++ over the first).

No compute calls: these run without a GPU."""
import ctypes as C
import glob
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "hsi-detectors-cuda_b200", "hsi_b200", "libhsi_b200.so")
CXXLIB = os.path.join(REPO, "hsi-detectors-cuda_b200", "hsi_b200", "libhsi_cxx.so")
LIB_OF_HEADER = {"hsi_b200.h": LIB, "hsi_batch.h": CXXLIB, "hsi_lagged.h": CXXLIB}


def declared_symbols(header=None):
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        if header and os.path.basename(h) != header:
            continue
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"HSI_API\s+[\w\s\*]+?\b(hsi_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "hsi_score_frames" in names and "hsi_detect" in names and len(names) >= 9


def test_every_header_is_mapped_to_its_library():
    headers = {os.path.basename(h) for h in glob.glob(os.path.join(REPO, "include", "*.h"))}
    assert headers == set(LIB_OF_HEADER)


@pytest.mark.parametrize("header", sorted(LIB_OF_HEADER))
def test_library_exports_every_declared_symbol(header):
    path = LIB_OF_HEADER[header]
    if not os.path.exists(path):
        pytest.fail(f"{path} not built (run `make -C hsi-detectors-cuda_b200`)")
    C.CDLL(LIB)  # libhsi_cxx resolves against it
    lib = C.CDLL(path)
    missing = [n for n in declared_symbols(header) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_host_only_entry_points_work_without_a_gpu():
    import hsi_b200
    assert hsi_b200.version() >= 100
    assert hsi_b200.plane_stride(520, 696) == 361920
    assert hsi_b200.plane_stride(3, 5) == 32
    assert hsi_b200.plane_stride(0, 5) == 0
    assert "positive definite" in hsi_b200.status_string(hsi_b200.E_NOT_POSITIVE_DEFINITE)
    sc = hsi_b200.scene(113, n_targets=8)
    spectra = hsi_b200.scene_spectra(sc)
    assert spectra.shape == (6 + 8 + 1, 113) and spectra.min() >= 0
    assert hsi_b200.detect_workspace_bytes(1024, 1024) > 0


def test_device_spectra_match_oracle_spectra():
    """Host-side spectra are double-precision and must agree exactly with the
    oracle's generator (both come from csrc/synth.h)."""
    import numpy as np
    import hsi_b200
    import oracle
    sc = hsi_b200.scene(64, n_targets=5, library_seed=1234)
    em, tg, an = oracle.scene_spectra(1234, 64, 6, 5)
    sp = hsi_b200.scene_spectra(sc)
    np.testing.assert_array_equal(sp[:6], em)
    np.testing.assert_array_equal(sp[6:11], tg)
    np.testing.assert_array_equal(sp[11], an)


def _fake_frame(hsi, **over):
    """A descriptor that passes host validation, with aligned device addresses
    that are never dereferenced (every case below fails validation first)."""
    base = 1 << 40
    f = hsi.Frame()
    f.cube, f.plane_stride, f.height, f.width, f.bands, f.dtype = base, 4096, 64, 64, 113, hsi.F16
    f.sam_targets, f.sam_norms, f.num_sam = base + 0x100000, base + 0x200000, 8
    f.num_cem, f.cem_weights = 8, base + 0x300000
    f.sam_best, f.sam_best_target, f.map_stride = base + 0x400000, base + 0x500000, 4096
    for k, v in over.items():
        setattr(f, k, v)
    return f


@pytest.mark.parametrize("bad", [
    dict(bands=0), dict(bands=257), dict(dtype=2), dict(height=0), dict(plane_stride=4000),
    dict(plane_stride=4100), dict(cube=(1 << 40) + 8), dict(num_sam=0, num_cem=0), dict(sam_targets=None),
    dict(sam_norms=None), dict(cem_weights=None), dict(sam_maps=1 << 41, map_stride=100),
    dict(num_sam=20, sam_best=None),
])
def test_batch_scoring_validates_every_descriptor_before_any_launch(bad):
    """hsi_score_frames_batch checks every host descriptor before it groups or
    launches anything: one bad frame among good ones fails the whole call with
    HSI_E_INVALID, so these run without a GPU."""
    import hsi_b200 as hsi
    L = hsi.lib()
    frames = [_fake_frame(hsi), _fake_frame(hsi, dtype=hsi.F32), _fake_frame(hsi, **bad)]
    arr = (hsi.Frame * len(frames))(*frames)
    assert L.hsi_score_frames_batch(C.cast(arr, C.c_void_p), len(frames), None, None) == hsi.E_INVALID
    assert L.hsi_score_frames_batch(None, 1, None, None) == hsi.E_INVALID
    assert L.hsi_score_frames_batch(C.cast(arr, C.c_void_p), 0, None, None) == hsi.E_INVALID


def test_screen_inference_validates_arguments_before_any_launch():
    """hsi_screen_infer / hsi_screen_infer_ctas reject bad arguments on the host,
    before any device call, so these run without a GPU."""
    import hsi_b200 as hsi
    L = hsi.lib()
    fake = C.c_void_p(1 << 40)  # 256-byte aligned, never dereferenced
    wb = L.hsi_screen_infer_workspace_bytes(113)
    assert wb > 0 and L.hsi_screen_infer_workspace_bytes(0) == 0
    args = lambda cube, dtype, stride, ws: (cube, 64, 96, 113, dtype, stride, fake, fake, fake, ws, wb)  # noqa: E731
    # a negative CTA cap, a missing cube, FP32 cubes, a plane stride short of the frame
    assert L.hsi_screen_infer_ctas(*args(fake, hsi.F16, 6144, fake), -1, None) == hsi.E_INVALID
    assert L.hsi_screen_infer_ctas(*args(None, hsi.F16, 6144, fake), 0, None) == hsi.E_INVALID
    assert L.hsi_screen_infer(*args(fake, hsi.F32, 6144, fake), None) == hsi.E_INVALID
    assert L.hsi_screen_infer_ctas(*args(fake, hsi.F16, 6000, fake), 8, None) == hsi.E_INVALID
    # no workspace
    assert L.hsi_screen_infer_ctas(*args(fake, hsi.F16, 6144, None), 8, None) == hsi.E_WORKSPACE


def test_statistics_sizes_and_host_side_rejections():
    """The FP64 statistics' host-side contract: the packed layout's size, the
    workspace (none up to 128 bands; both chains' matrices per frame above, which
    also covers the in-place path's target vectors), and the arguments rejected
    before any device call."""
    import hsi_b200 as hsi
    L = hsi.lib()
    tri = lambda n: n * (n + 1) // 2  # noqa: E731
    assert L.hsi_statistics_elements(113, 8) == 113 + 113 * 113 + 2 * 8 * 113 + 8
    for B in (1, 113, 124, 128):
        assert L.hsi_factor_workspace_bytes(3, B) == 0
    for B in (129, 224, 238, 239, 256):
        assert L.hsi_factor_workspace_bytes(3, B) == 8 * 4 * tri(B) * 3
        # per frame and chain the in-place path needs the target vectors (2 x 16 x B) and at
        # most the inverse's block-row buffer (16 x B) beside them, within 2 tri(B) doubles
        assert 2 * 16 * B + 16 * B <= 2 * tri(B)
    fake = C.c_void_p(1 << 40)
    call = lambda F, B, T, loading, ws, wsb: L.hsi_build_statistics(  # noqa: E731
        F, B, T, loading, fake, fake, 0, fake, None, None, fake, ws, wsb, None)
    assert call(1, 224, 16, 1e-6, None, 0) == hsi.E_WORKSPACE
    assert call(1, 224, 16, 1e-6, fake, L.hsi_factor_workspace_bytes(1, 224) - 1) == hsi.E_WORKSPACE
    assert call(0, 113, 8, 1e-6, None, 0) == hsi.E_INVALID
    assert call(1, 0, 8, 1e-6, None, 0) == hsi.E_INVALID
    assert call(1, 257, 8, 1e-6, None, 0) == hsi.E_INVALID
    assert call(1, 113, 65, 1e-6, None, 0) == hsi.E_INVALID
    assert call(1, 113, 8, -1.0, None, 0) == hsi.E_INVALID


def test_rx_ace_and_simt_reject_bad_frames_on_the_host():
    """RX/ACE entry points: band counts, targets, element types, strides and
    workspaces are checked before any device call.  The tensor-core path holds
    127 bands (more is HSI_E_CAPACITY: such frames take the plain path) and
    scores up to 64 targets in passes; the plain path takes 16 targets a call."""
    import hsi_b200 as hsi
    L = hsi.lib()
    fake = C.c_void_p(1 << 40)
    for name in ("simt", "tc"):
        fn = L.hsi_rx_ace_simt if name == "simt" else L.hsi_rx_ace
        wb = (L.hsi_rx_ace_simt_workspace_bytes if name == "simt" else L.hsi_rx_ace_workspace_bytes)(113, 8)
        assert wb > 0

        def call(cube=fake, B=113, dtype=hsi.F32, stride=6144, T=8, ws=fake, wsb=wb):
            return fn(cube, 64, 96, B, dtype, stride, fake, T, fake, fake, None, None, 6144, ws, wsb, None)

        assert call(cube=None) == hsi.E_INVALID
        assert call(B=0) == hsi.E_INVALID
        assert call(dtype=7) == hsi.E_INVALID
        assert call(stride=6000) == hsi.E_INVALID and call(stride=6148) == hsi.E_INVALID
        assert call(ws=None) == hsi.E_WORKSPACE and call(wsb=wb - 1) == hsi.E_WORKSPACE
        if name == "simt":
            assert call(B=257) == hsi.E_INVALID
            assert call(T=-1) == hsi.E_INVALID and call(T=17) == hsi.E_INVALID
        else:
            assert call(B=128) == hsi.E_CAPACITY and call(B=224) == hsi.E_CAPACITY
            assert call(T=-1) == hsi.E_CAPACITY and call(T=65) == hsi.E_CAPACITY


def test_detect_rejects_bad_jobs_on_the_host():
    """Detection: maps, counts, capacities, polarities and workspaces are checked
    before any device call."""
    import hsi_b200 as hsi
    L = hsi.lib()
    fake = C.c_void_p(1 << 40)
    wb = hsi.detect_workspace_bytes(64, 96)
    assert wb > 0

    def call(score=fake, count=fake, h=64, w=96, cap=16, out=fake, pol=hsi.LOWER_IS_BETTER, ws=fake, wsb=wb):
        return L.hsi_detect(score, None, h, w, C.c_float(0.1), 2, pol, cap, out, count, ws, wsb, None)

    assert call(score=None) == hsi.E_INVALID and call(count=None) == hsi.E_INVALID
    assert call(h=0) == hsi.E_INVALID and call(w=-1) == hsi.E_INVALID
    assert call(cap=-1) == hsi.E_INVALID and call(out=None) == hsi.E_INVALID
    assert call(pol=2) == hsi.E_INVALID
    assert call(ws=None) == hsi.E_WORKSPACE and call(wsb=wb - 1) == hsi.E_WORKSPACE
    assert call(ws=C.c_void_p((1 << 40) + 4)) == hsi.E_INVALID  # workspace not on 16 bytes


def test_moments_and_bip_reject_bad_frames_on_the_host():
    """Scene moments and the BIP scorer: frames, element types, strides,
    alignment, outputs and workspaces are checked before any device call."""
    import hsi_b200 as hsi
    L = hsi.lib()
    fake = C.c_void_p(1 << 40)

    def moments(fn=L.hsi_scene_moments, cube=fake, h=64, w=96, B=113, dtype=hsi.F32, stride=6144, out=fake,
                ws=fake, wsb=1 << 40):
        return fn(cube, h, w, B, dtype, stride, out, None, ws, wsb, None)

    assert moments(cube=None) == hsi.E_INVALID and moments(out=None) == hsi.E_INVALID
    assert moments(B=0) == hsi.E_INVALID and moments(B=257) == hsi.E_INVALID
    assert moments(dtype=3) == hsi.E_INVALID
    assert moments(stride=6000) == hsi.E_INVALID and moments(stride=6148) == hsi.E_INVALID
    assert moments(cube=C.c_void_p((1 << 40) + 8)) == hsi.E_INVALID  # cube not on 16 bytes
    assert moments(ws=None) == hsi.E_WORKSPACE and moments(wsb=16) == hsi.E_WORKSPACE
    assert moments(fn=L.hsi_scene_moments_tc, B=255) == hsi.E_CAPACITY  # past the limb GEMM's band views

    def bip(cube=fake, B=113, T=8, maps=fake, mstride=6144, best=fake):
        return L.hsi_sam_bip(cube, 64, 96, B, fake, fake, T, maps, mstride, best, None, None)

    assert bip(cube=None) == hsi.E_INVALID and bip(B=257) == hsi.E_INVALID
    assert bip(T=0) == hsi.E_INVALID and bip(T=65) == hsi.E_INVALID
    assert bip(maps=None, best=None) == hsi.E_INVALID  # nothing to write
    assert bip(mstride=6000) == hsi.E_INVALID
    assert bip(cube=C.c_void_p((1 << 40) + 2)) == hsi.E_INVALID  # not on 4 bytes


def test_conversions_and_gather_reject_bad_arguments_on_the_host():
    """Narrowing, the BIP transpose, demosaic and the candidates' gather check
    their arguments before any device call; narrowing nothing succeeds."""
    import hsi_b200 as hsi
    L = hsi.lib()
    fake = C.c_void_p(1 << 40)
    assert L.hsi_narrow_to_half(None, None, 0, None) == hsi.OK
    assert L.hsi_narrow_to_half(fake, fake, -1, None) == hsi.E_INVALID
    assert L.hsi_narrow_to_half(None, fake, 8, None) == hsi.E_INVALID
    assert L.hsi_narrow_to_half(C.c_void_p((1 << 40) + 4), fake, 8, None) == hsi.E_INVALID  # source not on 16 bytes
    assert L.hsi_transpose_bip_to_bsq(fake, None, 8, 8, 4, 64, None) == hsi.E_INVALID
    assert L.hsi_transpose_bip_to_bsq(fake, fake, 8, 8, 0, 64, None) == hsi.E_INVALID
    assert L.hsi_transpose_bip_to_bsq(fake, fake, 8, 8, 4, 63, None) == hsi.E_INVALID  # stride short of the frame
    # demosaic: more bands than mosaic cells, an unknown element type, a frame smaller than one period
    assert L.hsi_demosaic(fake, 64, 64, 4, 17, None, fake, hsi.F32, 256, None) == hsi.E_INVALID
    assert L.hsi_demosaic(fake, 64, 64, 4, 16, None, fake, 5, 256, None) == hsi.E_INVALID
    assert L.hsi_demosaic(fake, 3, 64, 4, 16, None, fake, hsi.F32, 256, None) == hsi.E_INVALID
    assert L.hsi_demosaic(fake, 64, 64, 4, 16, None, fake, hsi.F32, 255, None) == hsi.E_INVALID
    # gather: no candidate list, an output stride short of the capacity, an unknown element type
    assert L.hsi_gather_candidates(fake, hsi.F16, 4096, 113, 64, None, fake, 100, fake, 100, None) == hsi.E_INVALID
    assert L.hsi_gather_candidates(fake, hsi.F16, 4096, 113, 64, fake, fake, 100, fake, 99, None) == hsi.E_INVALID
    assert L.hsi_gather_candidates(fake, 4, 4096, 113, 64, fake, fake, 100, fake, 100, None) == hsi.E_INVALID
