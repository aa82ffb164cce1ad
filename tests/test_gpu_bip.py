"""GPU: hsi_sam_bip, SAM of a BIP cube with the transpose fused into the
scoring pass (the reference's SamVariant::BipDirect, src/sam.cu:80-125).

Its angle maps, best angles and best targets must be bit-identical to the BSQ
scorer (hsi_score_frames) on the transposed cube -- the same fmaf sequence per
pixel -- over band counts that do and do not divide the bank count, pixel
counts that leave a partial warp tile, and libraries of 1 to 40 targets (the
BSQ scorer takes three passes at 40); and within 5e-5 rad of the FP64 oracle
(the FP32 cosine's rounding, 2.2e-5 rad measured at 224 bands).
The reference's own test property (tests/test_sam.cpp: a pixel equal to a
target scores angle 0 for it) holds too, and C++ launch_sam_best(BipDirect)
routes here.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _vp(t):
    return C.c_void_p(t.data_ptr())


def _bip(hsi, H, W, B, T, seed):
    sc = hsi.scene(B, n_targets=max(T, 1), target_frac=0.01, library_seed=0x5EEDB000 + B, frame_seed=seed)
    cube, _ = hsi.generate(sc, H, W)  # BSQ at the library's plane stride
    P = H * W
    bip = cube[:, :P].t().contiguous()  # (P, B): pixel-major
    rng = np.random.default_rng(seed)
    lib = hsi.scene_targets(sc)
    if T > lib.shape[0]:
        extra = rng.uniform(0.05, 1.0, (T - lib.shape[0], B)).astype(np.float32)
        lib = np.concatenate([lib, extra])
    return cube, bip, lib[:T].copy()


@pytest.mark.parametrize("H,W,B,T,off", [(64, 96, 113, 8, 0), (37, 53, 113, 1, 0), (48, 40, 224, 16, 0),
                                         (33, 31, 16, 5, 0), (40, 64, 3, 2, 0), (50, 50, 128, 40, 0),
                                         (1, 7, 64, 3, 0), (29, 41, 30, 9, 0), (45, 47, 60, 12, 0),
                                         (20, 33, 250, 64, 0), (31, 29, 113, 8, 1), (31, 29, 64, 8, 1),
                                         (17, 19, 30, 3, 3)])
def test_bip_equals_bsq_bit_for_bit(hsi, orc, H, W, B, T, off):
    """Band counts of every row layout (odd, 2 mod 4, 4 mod 8, 0 mod 8), one
    to four target groups, and cubes whose base is not on 16 bytes (off
    floats into an allocation: the plain-load copies)."""
    bsq, bip, lib = _bip(hsi, H, W, B, T, seed=H * 1000 + W + B)
    if off:
        store = torch.zeros(bip.numel() + off, device="cuda")
        store[off:] = bip.reshape(-1)
        bip = store[off:]
    P = H * W
    tg = torch.from_numpy(lib).cuda()
    nr = torch.from_numpy(hsi.target_norms(lib)).cuda()
    want_maps = torch.empty((T, P), device="cuda")
    want_best = torch.empty(P, device="cuda")
    want_t = torch.empty(P, dtype=torch.int32, device="cuda")
    hsi.score_frames([hsi.make_frame(bsq, H, W, B, sam_targets=tg, sam_norms=nr, sam_maps=want_maps,
                                     sam_best=want_best, sam_best_target=want_t, map_stride=P)])
    maps = torch.full((T, P), -7.0, device="cuda")
    best = torch.full((P,), -7.0, device="cuda")
    bt = torch.full((P,), -7, dtype=torch.int32, device="cuda")
    st = hsi.lib().hsi_sam_bip(_vp(bip), H, W, B, _vp(tg), _vp(nr), T, _vp(maps), P, _vp(best), _vp(bt), None)
    assert st == 0, hsi.status_string(st)
    torch.cuda.synchronize()
    assert torch.equal(maps, want_maps)
    assert torch.equal(best, want_best)
    assert torch.equal(bt, want_t)
    f64, _ = orc.sam_best(bsq[:, :P].cpu().numpy(), lib)
    assert float(np.abs(best.cpu().numpy() - f64).max()) <= 5e-5


def test_bip_pixel_equal_to_a_target_scores_zero(hsi):
    H, W, B, T = 8, 8, 20, 3
    rng = np.random.default_rng(5)
    lib = rng.uniform(0.1, 1.0, (T, B)).astype(np.float32)
    bip = rng.uniform(0.1, 1.0, (H * W, B)).astype(np.float32)
    bip[10] = lib[2]
    bip[20] = 3.0 * lib[1]
    d = torch.from_numpy(bip).cuda()
    tg = torch.from_numpy(lib).cuda()
    nr = torch.from_numpy(hsi.target_norms(lib)).cuda()
    best = torch.empty(H * W, device="cuda")
    bt = torch.empty(H * W, dtype=torch.int32, device="cuda")
    assert hsi.lib().hsi_sam_bip(_vp(d), H, W, B, _vp(tg), _vp(nr), T, None, 0, _vp(best), _vp(bt), None) == 0
    torch.cuda.synchronize()
    b, t = best.cpu().numpy(), bt.cpu().numpy()
    assert b[10] < 1e-3 and t[10] == 2
    assert b[20] < 1e-3 and t[20] == 1


def test_bip_rejects_bad_arguments(hsi):
    L = hsi.lib()
    d = torch.zeros(64, device="cuda")
    vp = _vp(d)
    assert L.hsi_sam_bip(None, 4, 4, 4, vp, vp, 1, None, 0, vp, None, None) == hsi.E_INVALID
    assert L.hsi_sam_bip(vp, 4, 4, 4, vp, vp, 65, None, 0, vp, None, None) == hsi.E_INVALID
    assert L.hsi_sam_bip(vp, 4, 4, 4, vp, vp, 1, None, 0, None, None, None) == hsi.E_INVALID
    assert L.hsi_sam_bip(vp, 4, 4, 4, vp, vp, 1, vp, 15, None, None, None) == hsi.E_INVALID
