"""GPU: the batched frame runner (include/hsi_batch.h) on frames of uneven
sizes, band counts, element types and libraries, one of them a snapshot
mosaic demosaiced inside the run.

Checked: the CUDA-graph replay reproduces the eager run bit for bit; each
frame's SAM map matches the FP64 oracle (the scorer's tolerances: 1e-4 rad
away from zero angle, 2e-3 rad near it, where acos amplifies the FP32
cosine's rounding), its RX / ACE maps match
the single-frame path on the same statistics within the RX / ACE tolerance
(RX 1e-4 relative, ACE 1e-4 absolute: the autotuner may pick either RX path),
and its detection lists equal hsi_detect run on the batch's own maps.
"""
import numpy as np
import pytest
import torch

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


def test_batch_eager_graph_and_single_frame_agree(hsi, orc):
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
        want, _ = orc.sam_best(host, targets)
        err = np.abs(e["sam_best"].cpu().numpy() - want)
        assert err.max() <= 2e-3 and err[want > 0.05].max() <= 1e-4
        # RX / ACE against the single-frame path on the same statistics
        gm = hsi.scene_moments(cube, h, w, b, dtype=dt)
        s64, _, st = hsi.build_statistics(gm, b, torch.from_numpy(targets).cuda(), loading=1e-6)
        rx = torch.zeros(P, device="cuda")
        ace = torch.zeros(P, device="cuda")
        hsi.rx_ace(cube, h, w, b, s64[0], targets.shape[0], dtype=dt, rx=rx, ace_best=ace, simt=b > 127)
        torch.cuda.synchronize()
        r0 = rx.cpu().numpy()
        assert np.max(np.abs(e["rx"].cpu().numpy() - r0) / np.maximum(1.0, np.abs(r0))) <= 1e-4
        assert np.max(np.abs(e["ace_best"].cpu().numpy() - ace.cpu().numpy())) <= 1e-4
        # lists: hsi_detect on the batch's own maps
        maps = [(e["sam_best"], e["sam_target"], 0.12, hsi.LOWER_IS_BETTER),
                (e["ace_best"], e["ace_target"], 0.5, hsi.HIGHER_IS_BETTER),
                (e["rx"], None, e["rx_threshold"], hsi.HIGHER_IS_BETTER)]
        for k, (score, tgt, thr, pol) in enumerate(maps):
            count, lst = hsi.detect(score, tgt, h, w, thr, 2, pol, 2048)
            torch.cuda.synchronize()
            n = int(count.item())
            assert n == int(e["counts"][k].item()), (i, k)
            m = min(n, 2048)
            assert torch.equal(lst[:m], e["lists"][k][:m]), (i, k)
    batch.close()


def test_batch_rejects_bad_frames(hsi):
    t = np.ones((1, 8), np.float32)
    cube = torch.zeros((8, 64), device="cuda")
    with pytest.raises(hsi.HsiError):
        hsi.Batch([dict(cube=cube, height=0, width=8, bands=8, targets=t)])
    with pytest.raises(hsi.HsiError):
        hsi.Batch([dict(cube=cube, height=8, width=8, bands=8, targets=np.ones((17, 8), np.float32))])
