"""GPU parity: SAM / CEM filter-bank scoring against the FP64 oracle.

Cubes are generated on the device and read back, so both sides see the same
bits.  Tolerances (stated here, checked below):
  SAM angle  : |gpu - oracle| <= 2e-3 rad everywhere (the reference's own GPU
               gate, bench/bench_sam.cu:56) and <= 1e-4 rad where the angle is
               >= 0.02 rad (acos is ill-conditioned at 0);
  SAM label  : a different best target is allowed only where the oracle's
               angles of the two targets are within 2e-3 rad
               (bench/bench_sam.cu:156-183);
  CEM        : |gpu - oracle| <= 1e-5 * sum_b |w_b x_b| + 1e-6.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SAM_TOL = 2e-3
SAM_TOL_TIGHT = 1e-4


def _download(cube, B, P):
    return cube[:, :P].float().cpu().numpy().reshape(B, P)


def _check_sam(orc, host, targets, gpu_best, gpu_target, gpu_maps=None):
    T = targets.shape[0]
    allm = orc.sam_all(host, targets)
    best, which = orc.sam_best(host, targets)
    err = np.abs(gpu_best - best)
    assert err.max() <= SAM_TOL, f"max angle error {err.max()}"
    far = best >= 0.02
    if far.any():
        assert err[far].max() <= SAM_TOL_TIGHT, f"max angle error away from 0: {err[far].max()}"
    mism = np.nonzero(gpu_target != which)[0]
    for p in mism:
        g = gpu_target[p]
        assert 0 <= g < T
        assert abs(allm[g, p] - best[p]) <= SAM_TOL
    if gpu_maps is not None:
        merr = np.abs(gpu_maps - allm)
        assert merr.max() <= SAM_TOL
        if far.any():
            farm = allm >= 0.02
            assert merr[farm].max() <= SAM_TOL_TIGHT
    return err.max()


def _run(hsi, cube, H, W, B, dtype, sam=None, cem=None, maps=True):
    P = H * W
    dev = cube.device
    out = {}
    kw = {}
    if sam is not None:
        kw["sam_targets"] = torch.from_numpy(np.ascontiguousarray(sam, np.float32)).to(dev)
        kw["sam_norms"] = torch.from_numpy(hsi.target_norms(sam)).to(dev)
        out["sam_best"] = torch.full((P,), -7.0, device=dev)
        out["sam_best_target"] = torch.full((P,), -7, dtype=torch.int32, device=dev)
        if maps:
            out["sam_maps"] = torch.full((sam.shape[0], P), -7.0, device=dev)
    if cem is not None:
        kw["cem_weights"] = torch.from_numpy(np.ascontiguousarray(cem, np.float32)).to(dev)
        out["cem_best"] = torch.full((P,), -7.0, device=dev)
        out["cem_best_target"] = torch.full((P,), -7, dtype=torch.int32, device=dev)
        if maps:
            out["cem_maps"] = torch.full((cem.shape[0], P), -7.0, device=dev)
    f = hsi.make_frame(cube, H, W, B, dtype, map_stride=P, **kw, **out)
    hsi.score_frames([f])
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("dtype", [0, 1])
@pytest.mark.parametrize("T", [1, 4, 8])
def test_sam_generated_scene(hsi, orc, dtype, T):
    H, W, B = 52, 70, 113
    sc = hsi.scene(B, n_targets=T, target_frac=0.01, frame_seed=0x5EED0000 + T)
    cube, _ = hsi.generate(sc, H, W, dtype=dtype)
    host = _download(cube, B, H * W)
    targets = hsi.scene_targets(sc)
    r = _run(hsi, cube, H, W, B, dtype, sam=targets)
    _check_sam(orc, host, targets, r["sam_best"], r["sam_best_target"], r["sam_maps"])


@pytest.mark.parametrize("B", [1, 3, 16, 113, 127, 224, 256])
@pytest.mark.parametrize("shape", [(1, 1), (7, 13), (33, 17), (64, 64)])
def test_sam_shapes_and_band_counts(hsi, orc, B, shape):
    H, W = shape
    sc = hsi.scene(B, n_targets=3, target_frac=0.05, frame_seed=B * 1000 + H)
    cube, _ = hsi.generate(sc, H, W)
    host = _download(cube, B, H * W)
    targets = hsi.scene_targets(sc)
    r = _run(hsi, cube, H, W, B, 0, sam=targets)
    _check_sam(orc, host, targets, r["sam_best"], r["sam_best_target"], r["sam_maps"])


def test_sam_reference_cases(hsi, orc, golden):
    for name in ("identical", "zero", "best"):
        host = golden[f"case_{name}_cube"]
        targets = golden[f"case_{name}_targets"]
        B, H, W = host.shape
        stride = hsi.plane_stride(H, W)
        cube = torch.zeros((B, stride), device="cuda")
        cube[:, : H * W] = torch.from_numpy(host.reshape(B, -1)).cuda()
        r = _run(hsi, cube, H, W, B, 0, sam=targets)
        np.testing.assert_array_equal(r["sam_best_target"], golden[f"case_{name}_target"])
        assert np.max(np.abs(r["sam_best"] - golden[f"case_{name}_score"])) <= SAM_TOL
        assert not np.isnan(r["sam_best"]).any()
    # the orthogonal and the all-zero pixel are exactly pi/2 (no NaN)
    host = golden["case_zero_cube"]
    cube = torch.zeros((4, 32), device="cuda")
    cube[:, :2] = torch.from_numpy(host.reshape(4, -1)).cuda()
    r = _run(hsi, cube, 1, 2, 4, 0, sam=golden["case_zero_targets"])
    np.testing.assert_allclose(r["sam_best"], np.float32(np.pi / 2), atol=1e-6)


def test_sam_scale_invariance(hsi):
    rng = np.random.default_rng(7)
    t = rng.uniform(0.05, 1.0, (1, 16)).astype(np.float32)
    px = rng.uniform(0.05, 1.0, 16).astype(np.float32)
    gains = np.array([1.0, 0.01, 0.5, 3.0, 250.0], np.float32)
    host = (px[:, None] * gains[None, :]).astype(np.float32)
    cube = torch.zeros((16, 32), device="cuda")
    cube[:, :5] = torch.from_numpy(host).cuda()
    r = _run(hsi, cube, 1, 5, 16, 0, sam=t)
    assert np.max(np.abs(r["sam_best"] - r["sam_best"][0])) < 1e-4


def test_multi_pass_library(hsi, orc):
    """More than 16 targets: several passes, best carried through the outputs."""
    H, W, B = 40, 50, 64
    sc = hsi.scene(B, n_targets=20, target_frac=0.01, frame_seed=4)
    cube, _ = hsi.generate(sc, H, W)
    host = _download(cube, B, H * W)
    targets = hsi.scene_targets(sc)
    rng = np.random.default_rng(1)
    cem = rng.standard_normal((37, B)).astype(np.float32) * 0.1
    r = _run(hsi, cube, H, W, B, 0, sam=targets, cem=cem)
    _check_sam(orc, host, targets, r["sam_best"], r["sam_best_target"], r["sam_maps"])
    _check_cem(orc, host, cem, r)


def _check_cem(orc, host, cem, r):
    w64 = cem.astype(np.float64)
    stats = {"cem_weight": w64}
    best, which, allm = orc.cem(host, stats)
    mag = np.abs(w64) @ np.abs(host.astype(np.float64))
    tol = 1e-5 * mag + 1e-6
    assert (np.abs(r["cem_maps"] - allm) <= tol).all()
    assert (np.abs(r["cem_best"] - best) <= tol.max(axis=0)).all()
    mism = np.nonzero(r["cem_best_target"] != which)[0]
    for p in mism:
        g = r["cem_best_target"][p]
        assert abs(allm[g, p] - best[p]) <= 2 * tol[:, p].max()


@pytest.mark.parametrize("dtype", [0, 1])
def test_cem_with_scene_statistics(hsi, orc, dtype):
    H, W, B = 64, 64, 113
    sc = hsi.scene(B, n_targets=8, target_frac=0.002, frame_seed=0x5EED1001)
    cube, _ = hsi.generate(sc, H, W, dtype=dtype)
    host = _download(cube, B, H * W)
    targets = hsi.scene_targets(sc)
    s, o, n = orc.moments(host)
    st, S = orc.build_statistics(s, o, n, targets, 1e-6)
    assert st == 0
    cem = S["cem_weight"].astype(np.float32)
    r = _run(hsi, cube, H, W, B, dtype, sam=targets, cem=cem)
    _check_sam(orc, host, targets, r["sam_best"], r["sam_best_target"], r["sam_maps"])
    _check_cem(orc, host, cem, r)
    # against the FP64 weights themselves (what the statistics say the response is)
    best64, _, all64 = orc.cem(host, S)
    assert np.max(np.abs(r["cem_maps"] - all64)) < 1e-4


@pytest.mark.parametrize("max_sam,max_cem", [(4, 4), (8, 8), (8, 4)])
def test_sam_and_cem_banks_of_uneven_sizes(hsi, orc, max_sam, max_cem):
    """One device table whose frames carry fewer filters than the launch
    bounds (down to none of one kind): both banks are scored by one
    warpgroup, and empty slots must neither score nor write."""
    counts = [(max_sam, max_cem), (max_sam - 1, 0), (1, max_cem - 1), (0, max_cem)]
    frames, keep = [], []
    for i, (ns, nc) in enumerate(counts):
        H, W, B = 40 + i, 48, 113 - 20 * i
        sc = hsi.scene(B, n_targets=max(ns, nc, 1), target_frac=0.02, frame_seed=300 + i, library_seed=31 + i)
        cube, _ = hsi.generate(sc, H, W)
        lib = hsi.scene_targets(sc)
        P = H * W
        kw, out = {}, {}
        if ns:
            kw["sam_targets"] = torch.from_numpy(np.ascontiguousarray(lib[:ns])).cuda()
            kw["sam_norms"] = torch.from_numpy(hsi.target_norms(lib[:ns])).cuda()
            out["sam_best"] = torch.full((P,), -7.0, device="cuda")
            out["sam_best_target"] = torch.full((P,), -7, dtype=torch.int32, device="cuda")
            out["sam_maps"] = torch.full((ns, P), -7.0, device="cuda")
        cem = None
        if nc:
            rng = np.random.default_rng(40 + i)
            cem = (rng.standard_normal((nc, B)) / B).astype(np.float32)
            kw["cem_weights"] = torch.from_numpy(cem).cuda()
            out["cem_best"] = torch.full((P,), -7.0, device="cuda")
            out["cem_best_target"] = torch.full((P,), -7, dtype=torch.int32, device="cuda")
            out["cem_maps"] = torch.full((nc, P), -7.0, device="cuda")
        frames.append(hsi.make_frame(cube, H, W, B, 0, map_stride=P, **kw, **out))
        keep.append((cube, lib[:ns], cem, out, H, W, B, kw))
    table = hsi.frame_table(frames)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    hsi.score_frames_device(table, len(frames), max_bands=113, max_sam=max_sam, max_cem=max_cem, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    for cube, targets, cem, out, H, W, B, _ in keep:
        host = _download(cube, B, H * W)
        r = {k: v.cpu().numpy() for k, v in out.items()}
        if targets.shape[0]:
            _check_sam(orc, host, targets, r["sam_best"], r["sam_best_target"], r["sam_maps"])
        if cem is not None:
            _check_cem(orc, host, cem, r)


@pytest.mark.parametrize("B", [16, 113, 128])
@pytest.mark.parametrize("T", [(8, 8), (3, 0), (0, 5), (16, 16), (20, 9)])
def test_fp16_tensor_core_and_fma_scorers_match_the_oracle(hsi, orc, B, T):
    """FP16 cubes of at most 128 bands with host descriptors take the
    tensor-core scorer; descriptors in device memory take the FP32-FMA scorer.
    Both must meet the same tolerances against the FP64 oracle, including
    passes of more than 16 filters of a kind (20 SAM targets: two passes that
    carry the best), CEM weights of small magnitude (the per-filter power-of-two
    scale), and a last tile shorter than 128 pixels."""
    ns, nc = T
    H, W = 37, 101
    sc = hsi.scene(B, n_targets=max(ns, nc, 1), target_frac=0.03, frame_seed=500 + B + ns, library_seed=61 + nc)
    cube, _ = hsi.generate(sc, H, W, dtype=1)
    host = _download(cube, B, H * W)
    lib = hsi.scene_targets(sc)
    rng = np.random.default_rng(B + 7 * nc)
    cem = (rng.standard_normal((nc, B)) * 1e-3).astype(np.float32) if nc else None
    P = H * W
    for tensor_cores in (True, False):
        kw, out = {}, {}
        if ns:
            kw["sam_targets"] = torch.from_numpy(np.ascontiguousarray(lib[:ns])).cuda()
            kw["sam_norms"] = torch.from_numpy(hsi.target_norms(lib[:ns])).cuda()
            out["sam_best"] = torch.full((P,), -7.0, device="cuda")
            out["sam_best_target"] = torch.full((P,), -7, dtype=torch.int32, device="cuda")
            out["sam_maps"] = torch.full((ns, P), -7.0, device="cuda")
        if nc:
            kw["cem_weights"] = torch.from_numpy(cem).cuda()
            out["cem_best"] = torch.full((P,), -7.0, device="cuda")
            out["cem_best_target"] = torch.full((P,), -7, dtype=torch.int32, device="cuda")
            out["cem_maps"] = torch.full((nc, P), -7.0, device="cuda")
        frame = hsi.make_frame(cube, H, W, B, 1, map_stride=P, **kw, **out)
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        if tensor_cores:
            hsi.score_frames_batch([frame], status=status)
        else:
            hsi.score_frames_device(hsi.frame_table([frame]), 1, max_bands=B, max_sam=ns, max_cem=nc, dtype=1,
                                    status=status)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        r = {k: v.cpu().numpy() for k, v in out.items()}
        if ns:
            _check_sam(orc, host, lib[:ns], r["sam_best"], r["sam_best_target"], r["sam_maps"])
        if nc:
            _check_cem(orc, host, cem, r)


def test_batch_entry_mixes_element_types(hsi, orc):
    """One hsi_score_frames_batch call with FP32 and FP16 frames of several band
    counts (FP16 above 128 bands falls back to the FP32-FMA scorer)."""
    specs = [(113, 0), (113, 1), (224, 1), (16, 1), (60, 0)]
    frames, keep = [], []
    for i, (B, dt) in enumerate(specs):
        H, W = 50, 70 + 3 * i
        sc = hsi.scene(B, n_targets=4, target_frac=0.02, frame_seed=900 + i, library_seed=70 + i)
        cube, _ = hsi.generate(sc, H, W, dtype=dt)
        lib = hsi.scene_targets(sc)
        P = H * W
        best = torch.full((P,), -7.0, device="cuda")
        bt = torch.full((P,), -7, dtype=torch.int32, device="cuda")
        maps = torch.full((4, P), -7.0, device="cuda")
        # descriptors hold raw pointers: every tensor they name stays referenced until the scorer is done
        d_lib = torch.from_numpy(lib).cuda()
        d_norms = torch.from_numpy(hsi.target_norms(lib)).cuda()
        frames.append(hsi.make_frame(cube, H, W, B, dt, sam_targets=d_lib, sam_norms=d_norms, sam_maps=maps,
                                     sam_best=best, sam_best_target=bt, map_stride=P))
        keep.append((cube, lib, best, bt, maps, H, W, B, d_lib, d_norms))
    hsi.score_frames_batch(frames)
    torch.cuda.synchronize()
    for cube, lib, best, bt, maps, H, W, B, _, _ in keep:
        host = _download(cube, B, H * W)
        _check_sam(orc, host, lib, best.cpu().numpy(), bt.cpu().numpy(), maps.cpu().numpy())


def test_batched_frames_inline_and_device_table(hsi, orc):
    shapes = [(30, 41, 113), (64, 32, 16), (17, 19, 224)]
    frames, keep = [], []
    for i, (H, W, B) in enumerate(shapes):
        sc = hsi.scene(B, n_targets=3 + i, target_frac=0.02, frame_seed=77 + i, library_seed=5 + i)
        cube, _ = hsi.generate(sc, H, W)
        targets = hsi.scene_targets(sc)
        P = H * W
        tg = torch.from_numpy(targets).cuda()
        nr = torch.from_numpy(hsi.target_norms(targets)).cuda()
        best = torch.zeros(P, device="cuda")
        bt = torch.zeros(P, dtype=torch.int32, device="cuda")
        maps = torch.zeros((targets.shape[0], P), device="cuda")
        frames.append(hsi.make_frame(cube, H, W, B, 0, sam_targets=tg, sam_norms=nr, sam_maps=maps,
                                     sam_best=best, sam_best_target=bt, map_stride=P))
        keep.append((cube, targets, tg, nr, best, bt, maps, H, W, B))
    hsi.score_frames(frames)
    torch.cuda.synchronize()
    for cube, targets, _, _, best, bt, maps, H, W, B in keep:
        host = _download(cube, B, H * W)
        _check_sam(orc, host, targets, best.cpu().numpy(), bt.cpu().numpy(), maps.cpu().numpy())
        best.zero_()
        bt.zero_()
        maps.zero_()
    table = hsi.frame_table(frames)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    hsi.score_frames_device(table, len(frames), max_bands=224, max_sam=5, max_cem=0, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    for cube, targets, _, _, best, bt, maps, H, W, B in keep:
        host = _download(cube, B, H * W)
        _check_sam(orc, host, targets, best.cpu().numpy(), bt.cpu().numpy(), maps.cpu().numpy())


def test_device_table_rejects_frames_outside_bounds(hsi):
    """A frame with more bands than the launch allows is skipped, not overrun."""
    H, W, B = 8, 8, 64
    sc = hsi.scene(B, n_targets=2)
    cube, _ = hsi.generate(sc, H, W)
    t = torch.from_numpy(hsi.scene_targets(sc)).cuda()
    nr = torch.from_numpy(hsi.target_norms(hsi.scene_targets(sc))).cuda()
    best = torch.full((H * W,), -7.0, device="cuda")
    f = hsi.make_frame(cube, H, W, B, 0, sam_targets=t, sam_norms=nr, sam_best=best)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    hsi.score_frames_device(hsi.frame_table([f]), 1, max_bands=32, max_sam=2, max_cem=0, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == hsi.E_INVALID
    assert (best == -7.0).all()


def test_invalid_arguments_are_rejected(hsi):
    cube = torch.zeros((4, 32), device="cuda")
    t = np.ones((1, 4), np.float32)
    tg = torch.from_numpy(t).cuda()
    nr = torch.ones(1, device="cuda")
    best = torch.zeros(16, device="cuda")
    f = hsi.make_frame(cube, 4, 4, 4, 0, stride=30, sam_targets=tg, sam_norms=nr, sam_best=best)
    with pytest.raises(hsi.HsiError) as e:
        hsi.score_frames([f])
    assert e.value.status == hsi.E_INVALID
    f = hsi.make_frame(cube, 4, 4, 300, 0, sam_targets=tg, sam_norms=nr, sam_best=best)
    with pytest.raises(hsi.HsiError):
        hsi.score_frames([f])
