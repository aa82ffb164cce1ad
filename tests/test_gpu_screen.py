"""GPU: the learned screen against the FP64 oracle MLP (oracle/hsi_oracle.c,
itself pinned by finite differences in test_oracle_mlp.py).

Tolerances (stated here):
  gradients  per tensor |g - g64| / |g64| <= 2e-3 (FP32 accumulation over the
             batch against FP64, the same bfloat16-rounded weights, features
             and hidden activations on both sides), loss 1e-5 relative;
  logits     tensor-core inference against the oracle on the unrounded
             features: mean |error| <= 2e-3 and max <= 2e-2 of the largest
             |logit| (bfloat16 rounding of h1 lands on the other side of a tie
             for a few units; the first layer folds the normaliser into fp16
             weights, exact because its scales are powers of two).
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).float().numpy()


def _params(hsi, B, seed):
    L = hsi.lib()
    n = L.hsi_screen_param_count(B)
    p = torch.zeros(n, device="cuda")
    assert L.hsi_screen_init(_p(p), B, seed, None) == 0
    # non-zero biases so that every path of the backward pass is exercised
    g = torch.Generator(device="cuda").manual_seed(seed)
    Bp = (B + 63) // 64 * 64
    off_b1 = 64 * Bp
    p[off_b1:off_b1 + 64] = 0.1 * torch.randn(64, generator=g, device="cuda")
    p[off_b1 + 64 + 2048:off_b1 + 64 + 2048 + 32] = 0.1 * torch.randn(32, generator=g, device="cuda")
    p[-1] = -0.5
    return p, Bp


@pytest.mark.parametrize("B,n", [(113, 1000), (224, 513), (16, 64)])
def test_gradients_match_oracle(hsi, orc, B, n):
    L = hsi.lib()
    p, Bp = _params(hsi, B, 11 + B)
    rng = np.random.default_rng(B)
    feats = np.zeros((Bp, n), np.float32)
    feats[:B] = _bf16(rng.standard_normal((B, n)) * 1.5)
    labels = (rng.random(n) < 0.2).astype(np.float32)
    X = torch.from_numpy(feats).cuda()
    y = torch.from_numpy(labels).cuda()
    grads = torch.zeros_like(p)
    loss = torch.zeros(1, device="cuda")
    wb = L.hsi_screen_train_workspace_bytes(B, n)
    ws = torch.empty(wb, dtype=torch.uint8, device="cuda")
    assert L.hsi_screen_gradients(_p(p), B, _p(X), _p(y), n, C.c_float(3.0), _p(grads), _p(loss), _p(ws), wb,
                                  None) == 0
    torch.cuda.synchronize()
    _, loss0, g0 = orc.mlp(p.cpu().numpy(), B, feats[:B].T.copy(), labels, pos_weight=3.0, round_bf16=True,
                           grads=True)
    g = grads.cpu().numpy().astype(np.float64)
    assert abs(float(loss.item()) - loss0) <= 1e-5 * abs(loss0)
    off = 0
    for name, size in (("W1", 64 * Bp), ("b1", 64), ("W2", 2048), ("b2", 32), ("w3", 32), ("b3", 1)):
        a, b = g[off:off + size], g0[off:off + size]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert err <= 2e-3, f"{name}: {err:.3e}"
        off += size


def test_adam_step_moves_against_the_gradient(hsi):
    L = hsi.lib()
    B = 16
    p, _ = _params(hsi, B, 5)
    g = torch.randn_like(p)
    state = torch.zeros(2 * p.numel(), device="cuda")
    before = p.clone()
    assert L.hsi_screen_adam(_p(p), _p(state), _p(g), B, C.c_float(1e-3), 1, None) == 0
    torch.cuda.synchronize()
    step = (p - before).cpu().numpy()
    # first Adam step: -lr * sign(g) (up to eps)
    assert np.allclose(step, -1e-3 * np.sign(g.cpu().numpy()), atol=1e-6)


@pytest.mark.parametrize("B,H,W", [(113, 64, 96), (224, 40, 100), (60, 17, 33)])
def test_inference_matches_oracle(hsi, orc, B, H, W):
    L = hsi.lib()
    p, Bp = _params(hsi, B, 21 + B)
    P = H * W
    stride = hsi.plane_stride(H, W)
    rng = np.random.default_rng(B + H)
    host = (0.3 + 0.1 * rng.standard_normal((B, P))).astype(np.float16)
    cube = torch.zeros((B, stride), dtype=torch.float16, device="cuda")
    cube[:, :P] = torch.from_numpy(host).cuda()
    mean = host.astype(np.float64).mean(axis=1).astype(np.float32)
    scale = np.exp2(np.rint(-np.log2(host.astype(np.float64).std(axis=1)))).astype(np.float32)
    norm = np.zeros(2 * Bp, np.float32)
    norm[:B] = mean
    norm[Bp:Bp + B] = scale
    d_norm = torch.from_numpy(norm).cuda()
    logits = torch.full((P,), np.nan, device="cuda")
    wb = L.hsi_screen_infer_workspace_bytes(B)
    ws = torch.empty(wb, dtype=torch.uint8, device="cuda")
    st = L.hsi_screen_infer(_p(cube), H, W, B, 1, stride, _p(d_norm), _p(p), _p(logits), _p(ws), wb, None)
    assert st == 0, hsi.status_string(st)
    # the same kernel on fewer CTAs (room left for other work beside it): the same logits
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for cap in (7, sms - 2):
        capped = torch.full((P,), np.nan, device="cuda")
        st = L.hsi_screen_infer_ctas(_p(cube), H, W, B, 1, stride, _p(d_norm), _p(p), _p(capped), _p(ws), wb, cap,
                                     None)
        assert st == 0, hsi.status_string(st)
        assert torch.equal(capped, logits), cap
    assert L.hsi_screen_infer_ctas(_p(cube), H, W, B, 1, stride, _p(d_norm), _p(p), _p(logits), _p(ws), wb, -1,
                                   None) == hsi.E_INVALID
    torch.cuda.synchronize()
    feats = ((host.astype(np.float64) - mean[:, None].astype(np.float64)) * scale[:, None]).T.astype(np.float32)
    want = orc.mlp(p.cpu().numpy(), B, feats, round_bf16=True)[0]
    got = logits.cpu().numpy().astype(np.float64)
    assert np.isfinite(got).all()
    err = np.abs(got - want)
    scale_l = max(np.abs(want).max(), 1e-6)
    assert err.mean() <= 2e-3 * scale_l and err.max() <= 2e-2 * scale_l, (err.mean(), err.max(), scale_l)


def test_inference_rejects_fp32_cubes(hsi):
    L = hsi.lib()
    cube = torch.zeros((16, 64), device="cuda")
    p = torch.zeros(L.hsi_screen_param_count(16), device="cuda")
    ws = torch.empty(L.hsi_screen_infer_workspace_bytes(16), dtype=torch.uint8, device="cuda")
    out = torch.zeros(64, device="cuda")
    assert L.hsi_screen_infer(_p(cube), 8, 8, 16, 0, 64, _p(out), _p(p), _p(out), _p(ws), ws.numel(),
                              None) == hsi.E_INVALID
