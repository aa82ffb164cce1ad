"""GPU: the batched frame runner (include/hsi_batch.h) on frames of uneven
sizes, band counts, element types and libraries, one of them a snapshot
mosaic demosaiced inside the run.

Checked: the CUDA-graph replay reproduces the eager run bit for bit; each
frame's SAM map matches the FP64 oracle (the scorer's tolerances: 1e-4 rad
away from zero angle, 2e-3 rad near it, where acos amplifies the FP32
cosine's rounding); its RX / ACE maps match the FP64 oracle on the frame's
own FP64 statistics (RX 1e-4 relative, ACE 1e-4 absolute, whichever RX path
the autotuner picked); and its SAM, ACE and RX lists equal the oracle's
detect on the oracle's maps under the detection-set parity rule of
tests/parity.py (SAM 2e-3 rad -- the scorer's bound near zero angle --,
ACE 1e-4, RX 1e-4 of the value).
"""
import numpy as np
import pytest
import torch

import oracle
import parity

pytestmark = pytest.mark.gpu


def _mosaic(cube, bands, h, w, period):
    """Inverse of the demosaic: raw[y*p + oy, x*p + ox] = band (oy*p + ox) of pixel (x, y)."""
    c = cube[:, :h * w].reshape(bands, h, w)
    raw = torch.zeros((h * period, w * period), device=cube.device)
    for b in range(bands):
        oy, ox = divmod(b, period)
        raw[oy::period, ox::period] = c[b]
    return raw


def _frames(hsi):
    specs = [(64, 80, 16, 0, 3, "mosaic"), (100, 130, 113, 0, 8, None), (48, 64, 224, 0, 16, None),
             (256, 300, 113, 1, 3, None), (40, 40, 60, 0, 1, None)]
    frames, hosts = [], []
    for i, (h, w, b, dt, t, kind) in enumerate(specs):
        sc = hsi.scene(b, n_targets=max(t, 1), target_frac=0.01, anomaly_frac=0.002, library_seed=0x5EED6000 + i,
                       frame_seed=0x5EED6100 + i)
        cube, _ = hsi.generate(sc, h, w, dtype=dt)
        targets = hsi.scene_targets(sc)[:t]
        if kind == "mosaic":
            raw = _mosaic(cube, b, h, w, 4)
            frames.append(dict(raw=raw, period=4, bands=b, targets=targets))
        else:
            frames.append(dict(cube=cube, height=h, width=w, bands=b, dtype=dt, targets=targets))
        hosts.append((cube, h, w, b, dt, targets))
    return frames, hosts


def _collect(hsi, batch, hosts):
    out = []
    for i, (_, h, w, b, dt, t) in enumerate(hosts):
        o = batch.outputs(i)
        P = h * w
        d = {k: hsi.device_copy(getattr(o, k), P, torch.float32 if k in ("sam_best", "rx", "ace_best") else torch.int32)
             for k in ("sam_best", "sam_target", "rx", "ace_best", "ace_target")}
        d["counts"] = hsi.device_copy(o.counts, 3, torch.int32)
        d["lists"] = [hsi.device_copy(o.detections[k], 4 * batch.capacity, torch.int32).reshape(-1, 4) for k in range(3)]
        d["status"] = int(hsi.device_copy(o.status, 1, torch.int32).item())
        d["rx_threshold"] = o.rx_threshold
        out.append(d)
    return out


def test_batch_eager_graph_and_oracle_agree(hsi, orc):
    frames, hosts = _frames(hsi)
    batch = hsi.Batch(frames, sam_threshold=0.12, capacity=2048, autotune=True)
    stream = torch.cuda.Stream()
    batch.run(stream)
    stream.synchronize()
    eager = _collect(hsi, batch, hosts)
    batch.capture(stream)
    batch.launch(stream)
    batch.launch(stream)
    stream.synchronize()
    graph = _collect(hsi, batch, hosts)
    tuning = batch.tuning()
    assert tuning["tensor_core_rx_frames"] + tuning["plain_rx_frames"] == len(frames)
    for i, (cube, h, w, b, dt, targets) in enumerate(hosts):
        e, g = eager[i], graph[i]
        assert e["status"] == 0
        for k in ("sam_best", "sam_target", "rx", "ace_best", "ace_target", "counts"):
            assert torch.equal(e[k], g[k]), (i, k)
        P = h * w
        host = cube[:, :P].float().cpu().numpy()
        # SAM against the FP64 oracle
        want, which_sam = orc.sam_best(host, targets)
        err = np.abs(e["sam_best"].cpu().numpy() - want)
        assert err.max() <= 2e-3 and err[want > 0.05].max() <= 1e-4
        # RX / ACE against the FP64 oracle on the frame's FP64 statistics
        st, S = orc.build_statistics(*orc.moments(host), targets, 1e-6)
        assert st == 0
        best0, which0, rx0, all0 = orc.ace(host, S)
        rx_g = e["rx"].cpu().numpy()
        assert np.max(np.abs(rx_g - rx0) / np.maximum(1.0, np.abs(rx0))) <= 1e-4
        assert np.max(np.abs(e["ace_best"].cpu().numpy() - best0)) <= 1e-4
        # lists against the oracle's detect on the oracle's maps
        sam_all = orc.sam_all(host, targets)
        oracle_maps = [(want, which_sam, 0.12, False, 2e-3, parity.best_margin(sam_all, False), False),
                       (best0, which0, 0.5, True, 1e-4, parity.best_margin(all0, True), False),
                       (rx0, None, float(e["rx_threshold"]), True, 1e-4, None, True)]
        for k, (score, which, thr, higher, tol, margin, rel) in enumerate(oracle_maps):
            n = int(e["counts"][k].item())
            assert n <= 2048, (i, k)
            lst = e["lists"][k][:n].cpu().numpy()
            got = np.zeros(n, oracle.DETECTION_DTYPE)
            got["x"], got["y"], got["target"] = lst[:, 0], lst[:, 1], lst[:, 2]
            got["score"] = lst[:, 3].view(np.float32)
            _, ref = orc.detect(score, which, h, w, thr, 2, higher)
            parity.compare_lists(got, ref, score, h, w, thr, 2, tol, margin=margin, rel=rel)
    batch.close()


def test_batch_rejects_bad_frames(hsi):
    t = np.ones((1, 8), np.float32)
    cube = torch.zeros((8, 64), device="cuda")
    with pytest.raises(hsi.HsiError):
        hsi.Batch([dict(cube=cube, height=0, width=8, bands=8, targets=t)])
    with pytest.raises(hsi.HsiError):
        hsi.Batch([dict(cube=cube, height=8, width=8, bands=8, targets=np.ones((17, 8), np.float32))])
