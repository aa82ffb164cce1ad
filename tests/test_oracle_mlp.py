"""The FP64 screen-MLP oracle (no reference counterpart) pinned by central
finite differences of its own loss: analytic and numerical gradients agree to
1e-6 relative (FP64, bfloat16 rounding off, points away from ReLU kinks)."""
import numpy as np


def _setup(orc, B=12, n=24, seed=0):
    rng = np.random.default_rng(seed)
    P = orc.mlp_param_count(B)
    Bp = (B + 63) // 64 * 64
    p = (rng.standard_normal(P) * 0.3).astype(np.float32)
    W1 = p[:64 * Bp].reshape(64, Bp)
    W1[:, B:] = 0.0  # padding columns carry nothing
    x = rng.standard_normal((n, B)).astype(np.float32)
    y = (rng.random(n) < 0.3).astype(np.float32)
    return p, x, y, P, Bp


def test_mlp_gradient_matches_finite_differences(orc):
    B = 12
    p, x, y, P, Bp = _setup(orc, B)
    _, loss, g = orc.mlp(p, B, x, y, pos_weight=3.0, round_bf16=False, grads=True)
    rng = np.random.default_rng(1)
    # every bias, all of the last two layers, and a sample of W1 (inside the band range)
    offs = {"b1": 64 * Bp, "W2": 64 * Bp + 64, "b2": 64 * Bp + 64 + 2048, "w3": 64 * Bp + 64 + 2048 + 32,
            "b3": P - 1}
    idx = list(range(offs["b1"], P)) + [j * Bp + b for j, b in zip(rng.integers(0, 64, 60), rng.integers(0, B, 60))]
    h = np.float32(1e-4)  # small enough that no sample crosses a ReLU kink
    worst = 0.0
    for i in idx:
        q = p.copy()
        q[i] += h
        lp = orc.mlp(q, B, x, y, pos_weight=3.0, round_bf16=False)[1]
        q = p.copy()
        q[i] -= h
        lm = orc.mlp(q, B, x, y, pos_weight=3.0, round_bf16=False)[1]
        dq = float(np.float32(p[i] + h) - np.float32(p[i] - h))  # the step the float32 parameter took
        worst = max(worst, abs((lp - lm) / dq - g[i]) / max(1e-3, abs(g[i])))
    assert worst < 1e-6, worst


def test_mlp_padding_columns_get_no_gradient_and_rounding_is_bf16(orc):
    B = 12
    p, x, y, P, Bp = _setup(orc, B, seed=2)
    _, _, g = orc.mlp(p, B, x, y, round_bf16=True, grads=True)
    assert np.all(g[:64 * Bp].reshape(64, Bp)[:, B:] == 0.0)
    # with every weight already a bfloat16 value, rounding the weights changes nothing
    # except through h1, so logits differ only slightly
    a = orc.mlp(p, B, x, round_bf16=False)[0]
    b = orc.mlp(p, B, x, round_bf16=True)[0]
    assert np.max(np.abs(a - b)) < 0.05 * np.max(np.abs(a)) + 1e-6
