"""CPU oracles for the detection hot path - TEST INFRASTRUCTURE ONLY.

Two oracles, both loaded with ctypes:

* ``fp64``: this project's double-precision restatement (``hsi_oracle.c``).
  Detector statistics stay in double, so its maps are the FP64 truth that GPU
  error is stated against.
* ``ref``: the reference's own CPU scorer (src/sam_cpu.cpp,
  src/detectors_cpu.cpp, src/detector.cpp, src/linalg.cpp, ...), compiled
  unmodified into ``_ref/libhsi_ref.so`` by ``oracle/Makefile``.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this package, and only to check or to time the reference
CPU path.  The library under ``hsi-detectors-cuda_b200/`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FP64_LIB = os.path.join(HERE, "libhsi_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libhsi_ref.so")

DETECTION_DTYPE = np.dtype([("x", "<i4"), ("y", "<i4"), ("target", "<i4"), ("score", "<f4")])

STATS_OK = 0
STATS_EMPTY = 1
STATS_COVARIANCE_NOT_PD = 2
STATS_CORRELATION_NOT_PD = 3


class SceneSpec(C.Structure):
    """Mirror of ``hsi_scene_spec`` in csrc/synth.h."""

    _fields_ = [
        ("bands", C.c_int),
        ("n_end", C.c_int),
        ("n_targets", C.c_int),
        ("target_frac", C.c_float),
        ("anomaly_frac", C.c_float),
        ("noise_sigma", C.c_float),
        ("library_seed", C.c_uint64),
        ("frame_seed", C.c_uint64),
    ]


def build() -> None:
    """Compile both oracles (the reference one only where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


_f = lambda a: _ptr(a, C.c_float)  # noqa: E731
_d = lambda a: _ptr(a, C.c_double)  # noqa: E731
_i = lambda a: _ptr(a, C.c_int32)  # noqa: E731
_u8 = lambda a: _ptr(a, C.c_uint8)  # noqa: E731

_fp64 = None
_ref = None


def fp64_lib():
    global _fp64
    if _fp64 is None:
        if not os.path.exists(FP64_LIB):
            build()
        lib = C.CDLL(FP64_LIB)
        i64, f32p, f64p, i32p = C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int32)
        lib.orc_sam_all.argtypes = [f32p, i64, i64, C.c_int, f32p, f32p, C.c_int, f32p]
        lib.orc_sam_best.argtypes = [f32p, i64, i64, C.c_int, f32p, f32p, C.c_int, f32p, i32p]
        lib.orc_target_norms.argtypes = [f32p, C.c_int, C.c_int, f32p]
        lib.orc_detect.argtypes = [f32p, i32p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_void_p, i64]
        lib.orc_detect.restype = i64
        lib.orc_moments.argtypes = [f32p, i64, i64, C.c_int, f64p, f64p]
        lib.orc_moments_from_shifted.argtypes = [f64p, f64p, C.c_double, f64p, C.c_int, f64p, f64p]
        lib.orc_cholesky.argtypes = [f64p, C.c_int]
        lib.orc_cholesky.restype = C.c_int
        lib.orc_cholesky_solve.argtypes = [f64p, C.c_int, f64p, f64p]
        lib.orc_triangular_inverse_lower.argtypes = [f64p, C.c_int, f64p]
        lib.orc_build_statistics.argtypes = [f64p, f64p, C.c_double, C.c_int, f32p, C.c_int, C.c_double,
                                             f64p, f64p, f64p, f64p, f64p]
        lib.orc_build_statistics.restype = C.c_int
        lib.orc_rx.argtypes = [f32p, i64, i64, C.c_int, f64p, f64p, f32p]
        lib.orc_ace.argtypes = [f32p, i64, i64, C.c_int, f64p, f64p, f64p, f64p, C.c_int, f32p, i32p, f32p, f32p]
        lib.orc_cem.argtypes = [f32p, i64, i64, C.c_int, f64p, C.c_int, f32p, i32p, f32p]
        lib.orc_rx_threshold.argtypes = [C.c_int, C.c_double]
        lib.orc_rx_threshold.restype = C.c_double
        lib.orc_demosaic.argtypes = [f32p, C.c_int, C.c_int, C.c_int, C.c_int, i32p, f32p, i64]
        lib.orc_demosaic.restype = C.c_int
        lib.orc_scene_spectra.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, f32p, f32p, f32p]
        lib.orc_generate.argtypes = [C.POINTER(SceneSpec), i64, i64, i64, f32p, C.POINTER(C.c_uint8)]
        lib.orc_mlp_param_count.argtypes = [C.c_int]
        lib.orc_mlp_param_count.restype = i64
        lib.orc_mlp.argtypes = [f32p, C.c_int, f32p, f32p, C.c_int, C.c_double, C.c_int, f64p, f64p]
        lib.orc_mlp.restype = C.c_double
        _fp64 = lib
    return _fp64


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            build()
        lib = C.CDLL(REF_LIB)
        i64, f32p, f64p, i32p = C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int32)
        ci = C.c_int
        lib.ref_sam_best.argtypes = [f32p, ci, ci, ci, f32p, f32p, ci, f32p, i32p]
        lib.ref_sam_all.argtypes = [f32p, ci, ci, ci, f32p, f32p, ci, f32p]
        lib.ref_library_norms.argtypes = [f32p, ci, ci, f32p]
        lib.ref_detect.argtypes = [f32p, i32p, ci, ci, C.c_float, ci, ci, C.c_void_p, i64]
        lib.ref_detect.restype = i64
        lib.ref_moments.argtypes = [f32p, ci, ci, ci, f64p, f64p, f64p]
        lib.ref_build_statistics.argtypes = [f64p, f64p, C.c_double, ci, f32p, ci, C.c_double,
                                             f32p, f32p, f32p, f32p, f32p, C.c_char_p, ci]
        lib.ref_build_statistics.restype = ci
        lib.ref_rx.argtypes = [f32p, ci, ci, ci, f32p, f32p, f32p]
        lib.ref_rx.restype = ci
        lib.ref_ace_best.argtypes = [f32p, ci, ci, ci, ci, f32p, f32p, f32p, f32p, f32p, i32p, f32p]
        lib.ref_ace_best.restype = ci
        lib.ref_cem_best.argtypes = [f32p, ci, ci, ci, ci, f32p, f32p, f32p, f32p, i32p]
        lib.ref_cem_best.restype = ci
        lib.ref_rx_threshold.argtypes = [ci, C.c_double]
        lib.ref_rx_threshold.restype = C.c_double
        lib.ref_cholesky.argtypes = [f64p, ci]
        lib.ref_cholesky.restype = ci
        lib.ref_cholesky_solve.argtypes = [f64p, ci, f64p, f64p]
        lib.ref_triangular_inverse_lower.argtypes = [f64p, ci, f64p]
        lib.ref_moments_from_shifted.argtypes = [f64p, f64p, C.c_double, f64p, ci, f64p, f64p]
        lib.ref_demosaic.argtypes = [f32p, ci, ci, ci, ci, i32p, ci, f32p]
        lib.ref_demosaic.restype = ci
        lib.ref_synthetic_frame.argtypes = [ci, ci, ci, ci, ci, C.c_uint64, ci, f32p, C.POINTER(C.c_uint8), f32p]
        lib.ref_synthetic_frame.restype = ci
        lib.ref_frame_sam_cem.argtypes = [f32p, ci, ci, ci, f32p, ci, C.c_double, C.c_float, ci,
                                          f32p, f32p, i32p, f32p, i32p, C.c_void_p, i64]
        lib.ref_frame_sam_cem.restype = i64
        lib.ref_frame_rx_ace.argtypes = [f32p, ci, ci, ci, f32p, ci, C.c_double, f32p, i32p, f32p]
        lib.ref_frame_rx_ace.restype = ci
        lib.ref_read_envi.argtypes = [C.c_char_p, ci, i32p, f32p, i64, f32p, ci, C.c_char_p, ci]
        lib.ref_read_envi.restype = ci
        _ref = lib
    return _ref


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


# --------------------------------------------------------------------------
# FP64 restatement
# --------------------------------------------------------------------------

def target_norms(targets):
    t = _c(targets, np.float32)
    out = np.empty(t.shape[0], np.float32)
    fp64_lib().orc_target_norms(_f(t), t.shape[0], t.shape[1], _f(out))
    return out


def sam_best(cube, targets, norms=None):
    """cube: (B, H, W) or (B, P) float32 BSQ; targets (T, B)."""
    cube = _c(cube, np.float32)
    B = cube.shape[0]
    P = cube.size // B
    t = _c(targets, np.float32)
    n = target_norms(t) if norms is None else _c(norms, np.float32)
    score = np.empty(P, np.float32)
    which = np.empty(P, np.int32)
    fp64_lib().orc_sam_best(_f(cube), P, P, B, _f(t), _f(n), t.shape[0], _f(score), _i(which))
    return score, which


def sam_all(cube, targets, norms=None):
    cube = _c(cube, np.float32)
    B = cube.shape[0]
    P = cube.size // B
    t = _c(targets, np.float32)
    n = target_norms(t) if norms is None else _c(norms, np.float32)
    out = np.empty((t.shape[0], P), np.float32)
    fp64_lib().orc_sam_all(_f(cube), P, P, B, _f(t), _f(n), t.shape[0], _f(out))
    return out


def detect(score, target, height, width, threshold, nms_radius=2, higher_is_better=False,
           capacity=1 << 20):
    s = _c(score, np.float32).reshape(-1)
    tg = None if target is None else _c(target, np.int32).reshape(-1)
    out = np.zeros(capacity, DETECTION_DTYPE)
    n = fp64_lib().orc_detect(_f(s), _i(tg), height, width, threshold, nms_radius,
                              1 if higher_is_better else 0, out.ctypes.data, capacity)
    return n, out[: min(n, capacity)]


def moments(cube):
    cube = _c(cube, np.float32)
    B = cube.shape[0]
    P = cube.size // B
    s = np.empty(B, np.float64)
    o = np.empty((B, B), np.float64)
    fp64_lib().orc_moments(_f(cube), P, P, B, _d(s), _d(o))
    return s, o, float(P)


def build_statistics(sum_, outer, count, targets, loading):
    """Returns (status, dict of float64 arrays)."""
    sum_ = _c(sum_, np.float64)
    outer = _c(outer, np.float64)
    B = sum_.shape[0]
    t = np.zeros((0, B), np.float32) if targets is None else _c(targets, np.float32).reshape(-1, B)
    T = t.shape[0]
    out = {
        "mean": np.zeros(B), "whitener": np.zeros((B, B)), "target_white": np.zeros((T, B)),
        "target_norm2": np.zeros(T), "cem_weight": np.zeros((T, B)),
    }
    st = fp64_lib().orc_build_statistics(_d(sum_), _d(outer), count, B, _f(t), T, loading,
                                         _d(out["mean"]), _d(out["whitener"]), _d(out["target_white"]),
                                         _d(out["target_norm2"]), _d(out["cem_weight"]))
    return st, out


def rx(cube, stats):
    cube = _c(cube, np.float32)
    B = cube.shape[0]
    P = cube.size // B
    out = np.empty(P, np.float32)
    fp64_lib().orc_rx(_f(cube), P, P, B, _d(_c(stats["mean"], np.float64)),
                      _d(_c(stats["whitener"], np.float64)), _f(out))
    return out


def ace(cube, stats):
    """Returns (best score, best target, rx, per-target maps (T, P))."""
    cube = _c(cube, np.float32)
    B = cube.shape[0]
    P = cube.size // B
    T = stats["target_norm2"].shape[0]
    score = np.empty(P, np.float32)
    which = np.empty(P, np.int32)
    rxm = np.empty(P, np.float32)
    allm = np.empty((T, P), np.float32)
    fp64_lib().orc_ace(_f(cube), P, P, B, _d(_c(stats["mean"], np.float64)),
                       _d(_c(stats["whitener"], np.float64)), _d(_c(stats["target_white"], np.float64)),
                       _d(_c(stats["target_norm2"], np.float64)), T, _f(score), _i(which), _f(rxm), _f(allm))
    return score, which, rxm, allm


def cem(cube, stats):
    """Returns (best response, best target, per-target maps (T, P))."""
    cube = _c(cube, np.float32)
    B = cube.shape[0]
    P = cube.size // B
    T = stats["cem_weight"].shape[0]
    score = np.empty(P, np.float32)
    which = np.empty(P, np.int32)
    allm = np.empty((T, P), np.float32)
    fp64_lib().orc_cem(_f(cube), P, P, B, _d(_c(stats["cem_weight"], np.float64)), T, _f(score),
                       _i(which), _f(allm))
    return score, which, allm


def rx_threshold(bands, rate):
    return fp64_lib().orc_rx_threshold(bands, rate)


def demosaic(raw, period, bands, order=None):
    raw = _c(raw, np.float32)
    h, w = raw.shape
    oh, ow = h // period, w // period
    out = np.zeros((bands, oh, ow), np.float32)
    o = None if order is None else _c(order, np.int32)
    ok = fp64_lib().orc_demosaic(_f(raw), w, h, period, bands, _i(o), _f(out), oh * ow)
    return out if ok else None


def scene_spectra(library_seed, bands, n_end=6, n_targets=1):
    em = np.zeros((n_end, bands), np.float32)
    tg = np.zeros((max(n_targets, 1), bands), np.float32)
    an = np.zeros(bands, np.float32)
    fp64_lib().orc_scene_spectra(library_seed, bands, n_end, n_targets, _f(em), _f(tg), _f(an))
    return em, tg[:n_targets], an


def generate(spec: SceneSpec, height, width, pixel0=0):
    """Host-side scene: returns (cube (B, H, W) float32, truth (H, W) uint8)."""
    P = height * width
    cube = np.empty((spec.bands, height, width), np.float32)
    truth = np.empty((height, width), np.uint8)
    fp64_lib().orc_generate(C.byref(spec), pixel0, P, P, _f(cube), _u8(truth))
    return cube, truth


def scene(bands, n_targets=1, target_frac=0.005, anomaly_frac=0.0, library_seed=0x5EED0000,
          frame_seed=0x5EED0000, n_end=6, noise_sigma=0.005) -> SceneSpec:
    return SceneSpec(bands, n_end, n_targets, target_frac, anomaly_frac, noise_sigma, library_seed,
                     frame_seed)


# --------------------------------------------------------------------------
# Reference build (bit-faithful to the reference's CPU code)
# --------------------------------------------------------------------------

def ref_sam_best(cube, targets, norms):
    cube = _c(cube, np.float32)
    B, H, W = cube.shape
    t = _c(targets, np.float32)
    score = np.empty(H * W, np.float32)
    which = np.empty(H * W, np.int32)
    ref_lib().ref_sam_best(_f(cube), H, W, B, _f(t), _f(_c(norms, np.float32)), t.shape[0], _f(score), _i(which))
    return score, which


def ref_sam_all(cube, targets, norms):
    cube = _c(cube, np.float32)
    B, H, W = cube.shape
    t = _c(targets, np.float32)
    out = np.empty((t.shape[0], H * W), np.float32)
    ref_lib().ref_sam_all(_f(cube), H, W, B, _f(t), _f(_c(norms, np.float32)), t.shape[0], _f(out))
    return out


def ref_norms(targets):
    t = _c(targets, np.float32)
    out = np.empty(t.shape[0], np.float32)
    ref_lib().ref_library_norms(_f(t), t.shape[0], t.shape[1], _f(out))
    return out


def ref_detect(score, target, height, width, threshold, nms_radius=2, higher_is_better=False,
               capacity=1 << 20):
    s = _c(score, np.float32).reshape(-1)
    tg = None if target is None else _c(target, np.int32).reshape(-1)
    out = np.zeros(capacity, DETECTION_DTYPE)
    n = ref_lib().ref_detect(_f(s), _i(tg), height, width, threshold, nms_radius,
                             1 if higher_is_better else 0, out.ctypes.data, capacity)
    return n, out[: min(n, capacity)]


def ref_moments(cube):
    cube = _c(cube, np.float32)
    B, H, W = cube.shape
    s = np.empty(B, np.float64)
    o = np.empty((B, B), np.float64)
    cnt = np.zeros(1, np.float64)
    ref_lib().ref_moments(_f(cube), H, W, B, _d(s), _d(o), _d(cnt))
    return s, o, float(cnt[0])


def ref_build_statistics(sum_, outer, count, targets, loading):
    """Returns (ok, message, dict of float32 arrays) from the reference."""
    sum_ = _c(sum_, np.float64)
    outer = _c(outer, np.float64)
    B = sum_.shape[0]
    t = np.zeros((0, B), np.float32) if targets is None else _c(targets, np.float32).reshape(-1, B)
    T = t.shape[0]
    out = {
        "mean": np.zeros(B, np.float32), "whitener": np.zeros((B, B), np.float32),
        "target_white": np.zeros((T, B), np.float32), "target_norm2": np.zeros(T, np.float32),
        "cem_weight": np.zeros((T, B), np.float32),
    }
    err = C.create_string_buffer(512)
    ok = ref_lib().ref_build_statistics(_d(sum_), _d(outer), count, B, _f(t), T, loading,
                                        _f(out["mean"]), _f(out["whitener"]), _f(out["target_white"]),
                                        _f(out["target_norm2"]), _f(out["cem_weight"]), err, 512)
    return bool(ok), err.value.decode(), out


def ref_rx(cube, stats):
    cube = _c(cube, np.float32)
    B, H, W = cube.shape
    out = np.empty(H * W, np.float32)
    ok = ref_lib().ref_rx(_f(cube), H, W, B, _f(stats["mean"]), _f(stats["whitener"]), _f(out))
    return out if ok else None


def ref_ace_best(cube, stats):
    cube = _c(cube, np.float32)
    B, H, W = cube.shape
    T = stats["target_norm2"].shape[0]
    score = np.empty(H * W, np.float32)
    which = np.empty(H * W, np.int32)
    rxm = np.empty(H * W, np.float32)
    ok = ref_lib().ref_ace_best(_f(cube), H, W, B, T, _f(stats["mean"]), _f(stats["whitener"]),
                                _f(stats["target_white"]), _f(stats["target_norm2"]), _f(score),
                                _i(which), _f(rxm))
    return (score, which, rxm) if ok else None


def ref_cem_best(cube, stats):
    cube = _c(cube, np.float32)
    B, H, W = cube.shape
    T = stats["cem_weight"].shape[0]
    score = np.empty(H * W, np.float32)
    which = np.empty(H * W, np.int32)
    ok = ref_lib().ref_cem_best(_f(cube), H, W, B, T, _f(stats["mean"]), _f(stats["whitener"]),
                                _f(stats["cem_weight"]), _f(score), _i(which))
    return (score, which) if ok else None


def ref_rx_threshold(bands, rate):
    return ref_lib().ref_rx_threshold(bands, rate)


def ref_demosaic(raw, period, bands, order=None):
    raw = _c(raw, np.float32)
    h, w = raw.shape
    out = np.zeros((bands, h // period, w // period), np.float32)
    o = None if order is None else _c(order, np.int32)
    ok = ref_lib().ref_demosaic(_f(raw), w, h, period, bands, _i(o), 0 if o is None else len(o), _f(out))
    return out if ok else None


def ref_synthetic_frame(h, w, b, num_targets=3, target_radius=5, seed=4242, frame_index=0):
    cube = np.empty((b, h, w), np.float32)
    truth = np.empty((h, w), np.uint8)
    lib = np.empty((num_targets, b), np.float32)
    ok = ref_lib().ref_synthetic_frame(h, w, b, num_targets, target_radius, seed, frame_index,
                                       _f(cube), _u8(truth), _f(lib))
    return (cube, truth, lib) if ok else None


# ---------------------------------------------------------------------------
# learned screen (per-pixel MLP B -> 64 -> 32 -> 1)
# ---------------------------------------------------------------------------

def mlp_param_count(bands):
    return int(fp64_lib().orc_mlp_param_count(bands))


def mlp(params, bands, features, labels=None, pos_weight=1.0, round_bf16=True, grads=False):
    """FP64 forward (and, with labels, loss and gradient) of the screen MLP.
    features: (n, bands) float32.  Returns (logits, loss, grads or None)."""
    params = _c(params, np.float32)
    features = _c(features, np.float32)
    n = features.shape[0]
    logits = np.zeros(n, np.float64)
    g = np.zeros(mlp_param_count(bands), np.float64) if grads else None
    lab = None if labels is None else _c(labels, np.float32)
    loss = fp64_lib().orc_mlp(_f(params), bands, _f(features), _f(lab), n, float(pos_weight),
                              1 if round_bf16 else 0, _d(logits), _d(g))
    return logits, loss, g


def ref_read_envi(hdr_path, to=0):
    """The reference's own read_envi (oracle/_ref): (cube (H, W, B) float32 in the
    requested interleave's flat order, wavelengths) or raises RuntimeError with the
    reference's message."""
    lib = ref_lib()
    dims = np.zeros(4, np.int32)
    err = C.create_string_buffer(512)
    empty = np.zeros(1, np.float32)
    rc = lib.ref_read_envi(hdr_path.encode(), to, _i(dims), _f(empty), 0, _f(empty), 0, err, 512)
    if rc == 1:
        raise RuntimeError(err.value.decode())
    n = int(dims[0]) * int(dims[1]) * int(dims[2])
    data = np.zeros(max(n, 1), np.float32)
    wl = np.zeros(max(int(dims[3]), 1), np.float32)
    rc = lib.ref_read_envi(hdr_path.encode(), to, _i(dims), _f(data), n, _f(wl), int(dims[3]), err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode() if rc == 1 else "capacity")
    return (int(dims[0]), int(dims[1]), int(dims[2])), data[:n], wl[:int(dims[3])]
