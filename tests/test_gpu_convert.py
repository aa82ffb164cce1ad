"""GPU parity of the data-format kernels: demosaic (bit-exact against the
reference's own output in the golden fixtures, and against the oracle at
size), fp32 -> fp16 narrowing (bit-exact against round-to-nearest-even),
BIP -> BSQ transpose (exact), and the shifted-moment accumulation (FP64,
1e-12 relative)."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def _demosaic(hsi, raw, period, bands, order=None, dtype=0):
    h, w = raw.shape
    oh, ow = h // period, w // period
    stride = hsi.plane_stride(oh, ow)
    d_raw = torch.from_numpy(np.ascontiguousarray(raw, np.float32)).cuda()
    out = torch.zeros(bands * stride, dtype=torch.float32 if dtype == 0 else torch.float16, device="cuda")
    o = None if order is None else (C.c_int32 * bands)(*[int(v) for v in order])
    st = hsi.lib().hsi_demosaic(_p(d_raw), h, w, period, bands, o, _p(out), dtype, stride, None)
    assert st == 0, hsi.status_string(st)
    torch.cuda.synchronize()
    return out.float().cpu().numpy().reshape(bands, stride)[:, :oh * ow].reshape(bands, oh, ow)


def test_demosaic_matches_reference_fixtures(hsi, golden):
    raw, order = golden["demosaic_raw"], golden["demosaic_order"]
    assert np.array_equal(_demosaic(hsi, raw, 4, 16), golden["demosaic_16"])
    assert np.array_equal(_demosaic(hsi, raw, 4, 16, order), golden["demosaic_16_ordered"])
    assert np.array_equal(_demosaic(hsi, raw, 4, 15), golden["demosaic_15"])


@pytest.mark.parametrize("dtype", [0, 1])
def test_demosaic_at_size_matches_oracle(hsi, orc, dtype):
    rng = np.random.default_rng(3)
    raw = rng.random((1026, 1023), dtype=np.float32)  # ragged: trailing rows/columns dropped
    order = rng.permutation(16).astype(np.int32)
    got = _demosaic(hsi, raw, 4, 16, order, dtype)
    want = orc.demosaic(raw, 4, 16, order)
    if dtype == 0:
        assert np.array_equal(got, want)
    else:
        assert np.array_equal(got, want.astype(np.float16).astype(np.float32))


def test_demosaic_rejects_bad_orders(hsi):
    raw = torch.zeros((16, 16), device="cuda")
    out = torch.zeros(64 * 16, device="cuda")
    bad = (C.c_int32 * 4)(0, 1, 2, 16)
    assert hsi.lib().hsi_demosaic(_p(raw), 16, 16, 4, 4, bad, _p(out), 0, 16, None) == hsi.E_INVALID
    assert hsi.lib().hsi_demosaic(_p(raw), 16, 16, 4, 17, None, _p(out), 0, 16, None) == hsi.E_INVALID


def test_narrow_to_half_rounds_to_nearest_even(hsi):
    rng = np.random.default_rng(4)
    x = (rng.standard_normal(1_000_003) * 3).astype(np.float32)
    x[:6] = [0.0, -0.0, 65504.0, 1e-8, 2049.0, 2051.0]  # ties at 2049 / 2051 round to even
    src = torch.from_numpy(x).cuda()
    dst = torch.empty(x.size, dtype=torch.float16, device="cuda")
    assert hsi.lib().hsi_narrow_to_half(_p(src), _p(dst), x.size, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(dst.cpu().numpy().view(np.uint16), x.astype(np.float16).view(np.uint16))


def test_transpose_bip_to_bsq(hsi):
    H, W, B = 37, 101, 70
    rng = np.random.default_rng(5)
    bip = rng.random((H * W, B), dtype=np.float32)
    stride = hsi.plane_stride(H, W)
    src = torch.from_numpy(bip).cuda()
    dst = torch.full((B * stride,), -1.0, device="cuda")
    assert hsi.lib().hsi_transpose_bip_to_bsq(_p(src), _p(dst), H, W, B, stride, None) == 0
    torch.cuda.synchronize()
    got = dst.cpu().numpy().reshape(B, stride)
    assert np.array_equal(got[:, :H * W], bip.T)
    assert (got[:, H * W:] == -1.0).all()


def test_accumulate_shifted_moments(hsi, orc):
    B = 9
    rng = np.random.default_rng(6)
    x = rng.random((B, 500)).astype(np.float32)
    s, o, n = orc.moments(x)
    m = torch.from_numpy(np.concatenate([s, o.reshape(-1), [n]])).cuda()
    ref = rng.random(B).astype(np.float32)
    d_ref = torch.from_numpy(ref).cuda()
    s1 = torch.full((B,), 1.0, dtype=torch.float64, device="cuda")  # accumulates onto what is there
    s2 = torch.zeros((B, B), dtype=torch.float64, device="cuda")
    assert hsi.lib().hsi_accumulate_shifted_moments(_p(m), _p(d_ref), B, _p(s1), _p(s2), None) == 0
    torch.cuda.synchronize()
    d = x.astype(np.float64) - ref.astype(np.float64)[:, None]
    want1 = d.sum(axis=1) + 1.0
    want2 = np.tril(d @ d.T)
    assert np.allclose(s1.cpu().numpy(), want1, rtol=1e-12, atol=1e-9)
    got2 = s2.cpu().numpy()
    assert np.allclose(np.tril(got2), want2, rtol=1e-10, atol=1e-9)
    assert (np.triu(got2, 1) == 0).all()
