"""GPU: training the learned screen on the plain detector's decisions, and
what the trained screen gains over the method without it.

The labels are the plain tensor-core ACE detector's own decisions (best ACE >=
0.5) on synthetic 256 x 256 x 113 fp16 frames with 8 implanted targets.  The
screen trains on 10 frames; its proposal threshold is calibrated on the last
training frames for >= 99.9% recall; on three held-out frames the test then
measures:
  miss rate        plain-ACE detections the screen did not propose  (<= 1%)
  proposal share   pixels the plain detector must re-score          (<= 10%)
and the same for the untrained (initial) network calibrated the same way,
which must need at least 3x the proposals: that is the gain.  Re-scoring the
compacted proposals reproduces the full-frame ACE at those pixels exactly.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

H = W = 256
B, T = 113, 8
ACE_THRESHOLD = 0.5
LIB_SEED = 0x5EED4000


def _frame(hsi, lib_t, seed):
    sc = hsi.scene(B, n_targets=T, target_frac=0.004, anomaly_frac=0.001, library_seed=LIB_SEED, frame_seed=seed)
    cube, _ = hsi.generate(sc, H, W, dtype=1)
    gm = hsi.scene_moments(cube, H, W, B, dtype=1)
    s64, _, st = hsi.build_statistics(gm, B, lib_t, loading=1e-6)
    ace = torch.zeros(H * W, device="cuda")
    hsi.rx_ace(cube, H, W, B, s64[0], T, dtype=1, ace_best=ace, simt=False)
    norm = hsi.screen_normaliser(gm, B)
    torch.cuda.synchronize()
    assert int(st[0]) == 0
    return cube, ace, norm, s64[0]


def _calibrate(screen, hsi, frames):
    """Largest threshold keeping 99.9% of the positives of `frames`."""
    pos = []
    for cube, ace, norm, _ in frames:
        lg = screen.logits(cube, H, W, norm)
        pos.append(lg[ace >= ACE_THRESHOLD])
    pos = torch.cat(pos).sort().values
    k = int(np.floor(0.001 * pos.numel()))
    return float(pos[k].item()) - 1e-3


def _evaluate(screen, frames, thr):
    missed = positives = proposed = pixels = 0
    for cube, ace, norm, _ in frames:
        lg = screen.logits(cube, H, W, norm)
        p = ace >= ACE_THRESHOLD
        prop = lg >= thr
        positives += int(p.sum())
        missed += int((p & ~prop).sum())
        proposed += int(prop.sum())
        pixels += p.numel()
    return missed / max(positives, 1), proposed / pixels, positives


def test_trained_screen_gains_over_the_untrained(hsi):
    sc = hsi.scene(B, n_targets=T, library_seed=LIB_SEED)
    lib_t = torch.from_numpy(hsi.scene_targets(sc)).cuda()
    train = [_frame(hsi, lib_t, 0x5EED4001 + i) for i in range(10)]
    held = [_frame(hsi, lib_t, 0x5EED4101 + i) for i in range(3)]

    untrained = hsi.Screen(B, seed=7)
    screen = hsi.Screen(B, seed=7)
    loss0 = None
    for i, (cube, ace, norm, _) in enumerate(train):
        loss = screen.train_on(cube, H, W, 1, norm, ace, ACE_THRESHOLD, steps=120, batch=4096, seed=i)
        if loss0 is None:
            loss0 = float(loss.item())
    loss1 = float(loss.item())

    thr = _calibrate(screen, hsi, train[-3:])
    miss, share, npos = _evaluate(screen, held, thr)
    thr0 = _calibrate(untrained, hsi, train[-3:])
    miss0, share0, _ = _evaluate(untrained, held, thr0)
    print(f"loss {loss0:.4f} -> {loss1:.4f}; trained: miss {miss:.4%} proposals {share:.3%} ({npos} positives); "
          f"untrained: miss {miss0:.4%} proposals {share0:.3%}")
    assert loss1 < 0.5 * loss0
    assert npos > 500
    assert miss <= 0.01
    assert share <= 0.10
    assert share0 >= 3 * share


def test_rescoring_proposals_reproduces_the_full_frame_ace(hsi):
    sc = hsi.scene(B, n_targets=T, library_seed=LIB_SEED)
    lib_t = torch.from_numpy(hsi.scene_targets(sc)).cuda()
    cube, ace, norm, s64 = _frame(hsi, lib_t, 0x5EED4201)
    screen = hsi.Screen(B, seed=3)
    screen.train_on(cube, H, W, 1, norm, ace, ACE_THRESHOLD, steps=60, batch=2048)
    lg = screen.logits(cube, H, W, norm)
    thr = float(torch.quantile(lg, 0.9).item())
    cap = 1 << 14
    count, cand = hsi.detect(lg, None, H, W, thr, 0, hsi.HIGHER_IS_BETTER, cap)
    compact = hsi.gather_candidates(cube, 1, B, W, cand, count, cap)
    ace_c = torch.zeros(cap, device="cuda")
    hsi.rx_ace(compact, 1, cap, B, s64, T, dtype=1, ace_best=ace_c, simt=False)
    torch.cuda.synchronize()
    n = min(int(count.item()), cap)
    assert n > 0
    c = cand[:n].cpu().numpy()
    pix = torch.from_numpy(c[:, 1].astype(np.int64) * W + c[:, 0]).cuda()
    assert torch.equal(ace_c[:n], ace[pix])
