"""Python binding of libhsi_b200.so (the C ABI in include/hsi_b200.h).

A thin ctypes layer: torch tensors supply device memory and streams, every
computation runs in the library's sm_100a kernels.  There is no CPU fallback:
importing this module on a machine without the built library raises.

The functions mirror the reference's launch API for the detection path
(include/hsi/sam_cuda.hpp, detect_cuda.hpp, stats_cuda.hpp, detector.hpp in
GokulEdakkePuram/hsi-detectors-cuda): the same operations, argument meanings
and error behaviour (a non-zero status raises HsiError carrying the code).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libhsi_b200.so")

OK = 0
E_INVALID = 1
E_NOT_POSITIVE_DEFINITE = 10001
E_TIMEOUT = 10002
E_WORKSPACE = 10003
E_CAPACITY = 10004

F32 = 0
F16 = 1
LOWER_IS_BETTER = 0
HIGHER_IS_BETTER = 1
MAX_BANDS = 256
MAX_INLINE_FRAMES = 4
MAX_FILTERS_PER_PASS = 16


class HsiError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        text = _lib.hsi_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: status {status} ({text})" if what else f"status {status} ({text})")


class Scene(C.Structure):
    """hsi_scene: the synthetic scene model (csrc/synth.h)."""

    _fields_ = [
        ("bands", C.c_int32), ("n_end", C.c_int32), ("n_targets", C.c_int32),
        ("target_frac", C.c_float), ("anomaly_frac", C.c_float), ("noise_sigma", C.c_float),
        ("library_seed", C.c_uint64), ("frame_seed", C.c_uint64),
    ]


class DetectJob(C.Structure):
    """hsi_detect_job: one score map of a batched detection call (device pointers)."""

    _fields_ = [
        ("score", C.c_void_p), ("target", C.c_void_p), ("height", C.c_int32), ("width", C.c_int32),
        ("threshold", C.c_float), ("nms_radius", C.c_int32), ("polarity", C.c_int32), ("capacity", C.c_int32),
        ("out", C.c_void_p), ("count", C.c_void_p),
    ]


class Frame(C.Structure):
    """hsi_frame: one frame's cube, filter bank and output maps (device pointers)."""

    _fields_ = [
        ("cube", C.c_void_p), ("plane_stride", C.c_int64),
        ("height", C.c_int32), ("width", C.c_int32), ("bands", C.c_int32), ("dtype", C.c_int32),
        ("sam_targets", C.c_void_p), ("sam_norms", C.c_void_p), ("num_sam", C.c_int32),
        ("num_cem", C.c_int32), ("cem_weights", C.c_void_p),
        ("sam_maps", C.c_void_p), ("sam_best", C.c_void_p), ("sam_best_target", C.c_void_p),
        ("cem_maps", C.c_void_p), ("cem_best", C.c_void_p), ("cem_best_target", C.c_void_p),
        ("map_stride", C.c_int64),
    ]


DETECTION_BYTES = 16

_lib = None


def build(force: bool = False) -> None:
    """Compile the library for sm_100a with nvcc (cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-j8", "-C", PKG] + (["-B"] if force else []), check=True)


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG}` "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64 = C.c_void_p, C.c_int, C.c_int64
        L.hsi_status_string.argtypes = [i32]
        L.hsi_status_string.restype = C.c_char_p
        L.hsi_version.restype = i32
        L.hsi_plane_stride.argtypes = [i32, i32]
        L.hsi_plane_stride.restype = i64
        L.hsi_scene_spectra.argtypes = [C.POINTER(Scene), vp]
        L.hsi_scene_spectra.restype = i32
        L.hsi_generate.argtypes = [C.POINTER(Scene), vp, i32, i32, i64, vp, i32, i64, vp, vp]
        L.hsi_generate.restype = i32
        L.hsi_score_frames.argtypes = [C.POINTER(Frame), i32, vp]
        L.hsi_score_frames.restype = i32
        L.hsi_score_frames_device.argtypes = [vp, i32, i32, i32, i32, i32, vp, vp]
        L.hsi_score_frames_device.restype = i32
        L.hsi_detect_workspace_bytes.argtypes = [i32, i32]
        L.hsi_detect_workspace_bytes.restype = C.c_size_t
        L.hsi_detect.argtypes = [vp, vp, i32, i32, C.c_float, i32, i32, i32, vp, vp, vp, C.c_size_t, vp]
        L.hsi_detect.restype = i32
        L.hsi_detect_batch_workspace_bytes.argtypes = [C.POINTER(DetectJob), i32]
        L.hsi_detect_batch_workspace_bytes.restype = C.c_size_t
        L.hsi_detect_batch.argtypes = [C.POINTER(DetectJob), i32, vp, C.c_size_t, vp]
        L.hsi_detect_batch.restype = i32
        _optional_symbols(L)
        _lib = L
    return _lib


def _optional_symbols(L):
    """Entry points added after the first slice; bound when present."""
    vp, i32, i64, f64 = C.c_void_p, C.c_int, C.c_int64, C.c_double
    table = {
        "hsi_stats_workspace_bytes": ([i32, i32, i32], C.c_size_t),
        "hsi_scene_moments": ([vp, i32, i32, i32, i32, i64, vp, vp, vp, C.c_size_t, vp], i32),
        "hsi_scene_moments_simt": ([vp, i32, i32, i32, i32, i64, vp, vp, vp, C.c_size_t, vp], i32),
        "hsi_scene_moments_tc": ([vp, i32, i32, i32, i32, i64, vp, vp, vp, C.c_size_t, vp], i32),
        "hsi_score_frames_device_grid": ([vp, i32, i32, i32, i32, i32, vp, i32, vp], i32),
        "hsi_score_frames_batch": ([vp, i32, vp, vp], i32),
        "hsi_scene_moments_batch_workspace_bytes": ([C.POINTER(MomentsJob), i32], C.c_size_t),
        "hsi_scene_moments_batch": ([C.POINTER(MomentsJob), i32, vp, C.c_size_t, vp], i32),
        "hsi_statistics_elements": ([i32, i32], C.c_size_t),
        "hsi_factor_workspace_bytes": ([i32, i32], C.c_size_t),
        "hsi_build_statistics": ([i32, i32, i32, f64, vp, vp, i64, vp, vp, vp, vp, vp, C.c_size_t, vp], i32),
        "hsi_rx_ace_workspace_bytes": ([i32, i32], C.c_size_t),
        "hsi_rx_ace": ([vp, i32, i32, i32, i32, i64, vp, i32, vp, vp, vp, vp, i64, vp, C.c_size_t, vp], i32),
        "hsi_rx_ace_simt_workspace_bytes": ([i32, i32], C.c_size_t),
        "hsi_rx_ace_simt": ([vp, i32, i32, i32, i32, i64, vp, i32, vp, vp, vp, vp, i64, vp, C.c_size_t, vp], i32),
        "hsi_demosaic": ([vp, i32, i32, i32, i32, vp, vp, i32, i64, vp], i32),
        "hsi_narrow_to_half": ([vp, vp, i64, vp], i32),
        "hsi_transpose_bip_to_bsq": ([vp, vp, i32, i32, i32, i64, vp], i32),
        "hsi_accumulate_shifted_moments": ([vp, vp, i32, vp, vp, vp], i32),
        "hsi_detect_noalloc": ([vp, vp, i32, i32, C.c_float, i32, i32, i32, vp, vp, vp], i32),
        "hsi_screen_param_count": ([i32], i64),
        "hsi_screen_init": ([vp, i32, C.c_uint64, vp], i32),
        "hsi_screen_normaliser": ([vp, i32, vp, vp], i32),
        "hsi_screen_batch": ([vp, vp, i32, i32, i32, vp, C.c_float, C.c_uint64, i32, i32, vp, vp, vp], i32),
        "hsi_screen_gather": ([vp, i32, i64, i32, vp, vp, i32, vp, vp], i32),
        "hsi_screen_train_workspace_bytes": ([i32, i32], C.c_size_t),
        "hsi_screen_gradients": ([vp, i32, vp, vp, i32, C.c_float, vp, vp, vp, C.c_size_t, vp], i32),
        "hsi_screen_adam": ([vp, vp, vp, i32, C.c_float, i32, vp], i32),
        "hsi_screen_infer_workspace_bytes": ([i32], C.c_size_t),
        "hsi_screen_infer": ([vp, i32, i32, i32, i32, i64, vp, vp, vp, vp, C.c_size_t, vp], i32),
        "hsi_screen_infer_ctas": ([vp, i32, i32, i32, i32, i64, vp, vp, vp, vp, C.c_size_t, i32, vp], i32),
        "hsi_gather_candidates": ([vp, i32, i64, i32, i32, vp, vp, i32, vp, i64, vp], i32),
        "hsi_sam_bip": ([vp, i32, i32, i32, vp, vp, i32, vp, i64, vp, vp, vp], i32),
    }
    for name, (argtypes, restype) in table.items():
        if hasattr(L, name):
            fn = getattr(L, name)
            fn.argtypes = argtypes
            fn.restype = restype


def check(status: int, what: str = "") -> None:
    if status != OK:
        raise HsiError(status, what)


def status_string(status: int) -> str:
    return lib().hsi_status_string(status).decode()


def version() -> int:
    return lib().hsi_version()


def plane_stride(height: int, width: int) -> int:
    """Device plane stride (pixels rounded up to 32); the reference's bsq_plane_stride."""
    return lib().hsi_plane_stride(height, width)


# ---------------------------------------------------------------------------
# helpers over torch tensors
# ---------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def scene(bands, n_targets=1, target_frac=0.005, anomaly_frac=0.0, library_seed=0x5EED0000,
          frame_seed=0x5EED0000, n_end=6, noise_sigma=0.005) -> Scene:
    return Scene(bands, n_end, n_targets, target_frac, anomaly_frac, noise_sigma, library_seed, frame_seed)


def scene_spectra(sc: Scene):
    """Host numpy array (n_end + n_targets + 1, bands): endmembers, targets, anomaly."""
    import numpy as np
    out = np.zeros((sc.n_end + sc.n_targets + 1, sc.bands), np.float32)
    check(lib().hsi_scene_spectra(C.byref(sc), out.ctypes.data), "hsi_scene_spectra")
    return out


def scene_targets(sc: Scene):
    """The implanted library (n_targets, bands) as a host numpy array."""
    return scene_spectra(sc)[sc.n_end:sc.n_end + sc.n_targets].copy()


def generate(sc: Scene, height, width, dtype=F32, pixel0=0, stride=None, out=None, truth=True,
             device="cuda", stream=None):
    """Generate a frame on the device.  Returns (cube (bands, stride) tensor, truth (pixels,) uint8)."""
    torch = _torch()
    stride = plane_stride(height, width) if stride is None else stride
    tdt = torch.float32 if dtype == F32 else torch.float16
    if out is None:
        out = torch.zeros((sc.bands, stride), dtype=tdt, device=device)
    spectra = torch.from_numpy(scene_spectra(sc)).to(device)
    tr = torch.empty(height * width, dtype=torch.uint8, device=device) if truth else None
    check(lib().hsi_generate(C.byref(sc), _ptr(spectra), height, width, pixel0, _ptr(out), dtype, stride,
                             _ptr(tr), _stream(stream)), "hsi_generate")
    return out, tr


def target_norms(targets):
    """L2 norm of each target, accumulated in double then narrowed (SpectralLibrary::norms)."""
    import numpy as np
    t = np.asarray(targets, np.float64)
    return np.sqrt((t * t).sum(axis=1)).astype(np.float32)


def make_frame(cube, height, width, bands, dtype=F32, stride=None, sam_targets=None, sam_norms=None,
               cem_weights=None, sam_maps=None, sam_best=None, sam_best_target=None, cem_maps=None,
               cem_best=None, cem_best_target=None, map_stride=None) -> Frame:
    stride = cube.shape[-1] if stride is None else stride
    P = height * width
    f = Frame()
    f.cube = cube.data_ptr()
    f.plane_stride = stride
    f.height, f.width, f.bands, f.dtype = height, width, bands, dtype
    f.sam_targets = sam_targets.data_ptr() if sam_targets is not None else None
    f.sam_norms = sam_norms.data_ptr() if sam_norms is not None else None
    f.num_sam = 0 if sam_targets is None else sam_targets.shape[0]
    f.cem_weights = cem_weights.data_ptr() if cem_weights is not None else None
    f.num_cem = 0 if cem_weights is None else cem_weights.shape[0]
    for name, t in (("sam_maps", sam_maps), ("sam_best", sam_best), ("sam_best_target", sam_best_target),
                    ("cem_maps", cem_maps), ("cem_best", cem_best), ("cem_best_target", cem_best_target)):
        setattr(f, name, t.data_ptr() if t is not None else None)
    if map_stride is None:
        maps = sam_maps if sam_maps is not None else cem_maps
        map_stride = maps.shape[-1] if maps is not None else P
    f.map_stride = map_stride
    return f


def score_frames(frames, stream=None) -> None:
    """Score up to 4 frames whose descriptors live on the host (one launch per pass)."""
    n = len(frames)
    arr = (Frame * n)(*frames)
    check(lib().hsi_score_frames(arr, n, _stream(stream)), "hsi_score_frames")


def score_frames_batch(frames, status=None, stream=None) -> None:
    """Any number of frames with host descriptors (Frame structs): FP16 cubes of at
    most 128 bands on the tensor cores, the rest on the FP32-FMA scorer."""
    n = len(frames)
    arr = (Frame * n)(*frames)
    check(lib().hsi_score_frames_batch(C.cast(arr, C.c_void_p), n, _ptr(status), _stream(stream)),
          "hsi_score_frames_batch")


def frame_table(frames, device="cuda"):
    """Upload descriptors to a device table for hsi_score_frames_device."""
    torch = _torch()
    n = len(frames)
    arr = (Frame * n)(*frames)
    raw = bytes(arr)
    host = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
    return host.to(device)


def score_frames_device(table, num_frames, max_bands, max_sam, max_cem, dtype=F32, status=None,
                        stream=None) -> None:
    """Batched scoring from a device descriptor table (see frame_table).  `status`
    (device int32 tensor, optional) receives HSI_E_INVALID for frames outside the bounds."""
    check(lib().hsi_score_frames_device(_ptr(table), num_frames, dtype, max_bands, max_sam, max_cem,
                                        _ptr(status), _stream(stream)), "hsi_score_frames_device")


def detect_workspace_bytes(height, width) -> int:
    return lib().hsi_detect_workspace_bytes(height, width)


def detect(score, target, height, width, threshold, nms_radius=2, polarity=LOWER_IS_BETTER, capacity=4096,
           out=None, count=None, workspace=None, stream=None):
    """Threshold + NMS + raster-order compaction on the device.

    Returns (count tensor (1,) uint32-as-int32, detections (capacity, 4) int32 view).  The count is
    the number found (it may exceed capacity)."""
    torch = _torch()
    dev = score.device
    if out is None:
        out = torch.zeros((max(capacity, 1), 4), dtype=torch.int32, device=dev)
    if count is None:
        count = torch.zeros(1, dtype=torch.int32, device=dev)
    if workspace is None:
        workspace = torch.empty(detect_workspace_bytes(height, width), dtype=torch.uint8, device=dev)
    check(lib().hsi_detect(_ptr(score), _ptr(target), height, width, float(threshold), nms_radius, polarity,
                           capacity, _ptr(out), _ptr(count), _ptr(workspace), workspace.numel(),
                           _stream(stream)), "hsi_detect")
    return count, out


def detect_job(score, target, height, width, threshold, nms_radius, polarity, capacity, out, count) -> DetectJob:
    return DetectJob(score.data_ptr(), None if target is None else target.data_ptr(), height, width,
                     float(threshold), nms_radius, polarity, capacity, out.data_ptr(), count.data_ptr())


def detect_batch_workspace_bytes(jobs) -> int:
    arr = (DetectJob * len(jobs))(*jobs)
    return lib().hsi_detect_batch_workspace_bytes(arr, len(jobs))


def detect_batch(jobs, workspace, stream=None) -> None:
    """Up to 64 maps in three launches; see hsi_detect_batch."""
    arr = (DetectJob * len(jobs))(*jobs)
    check(lib().hsi_detect_batch(arr, len(jobs), _ptr(workspace), workspace.numel(), _stream(stream)),
          "hsi_detect_batch")


def detections_to_numpy(count, out, capacity):
    """Device detection list -> numpy structured array (x, y, target, score), clamped to capacity."""
    import numpy as np
    n = int(count.item()) & 0xFFFFFFFF
    k = min(n, capacity)
    raw = out[:k].cpu().numpy()
    dt = np.dtype([("x", "<i4"), ("y", "<i4"), ("target", "<i4"), ("score", "<f4")])
    return n, raw.view(dt).reshape(-1) if k > 0 else np.zeros(0, dt)


# ---------------------------------------------------------------------------
# scene statistics and FP64 factorisation
# ---------------------------------------------------------------------------

E_CORRELATION_NOT_PD = 10006
E_EMPTY = 10007


def stats_workspace_bytes(height, width, bands) -> int:
    return lib().hsi_stats_workspace_bytes(height, width, bands)


def moments_elements(bands) -> int:
    return bands + bands * bands + 1


def scene_moments(cube, height, width, bands, dtype=F32, stride=None, out=None, reference=None, workspace=None,
                  simt=False, path=None, stream=None):
    """Raw moments of one frame on the device: (B + B*B + 1,) float64 = sum, outer, count
    (the reference's SpectralMoments).  path: None (automatic), "simt" (plain FP32
    CUDA cores) or "tc" (integer tensor cores at any size)."""
    torch = _torch()
    dev = cube.device
    stride = cube.shape[-1] if stride is None else stride
    if out is None:
        out = torch.empty(moments_elements(bands), dtype=torch.float64, device=dev)
    if workspace is None:
        workspace = torch.empty(stats_workspace_bytes(height, width, bands), dtype=torch.uint8, device=dev)
    path = "simt" if simt else path
    fn = {None: lib().hsi_scene_moments, "simt": lib().hsi_scene_moments_simt,
          "tc": lib().hsi_scene_moments_tc}[path]
    check(fn(_ptr(cube), height, width, bands, dtype, stride, _ptr(out), _ptr(reference), _ptr(workspace),
             workspace.numel(), _stream(stream)), "hsi_scene_moments")
    return out


class MomentsJob(C.Structure):
    """hsi_moments_job: one frame of hsi_scene_moments_batch."""
    _fields_ = [("cube", C.c_void_p), ("plane_stride", C.c_int64), ("moments", C.c_void_p),
                ("reference", C.c_void_p), ("height", C.c_int32), ("width", C.c_int32), ("bands", C.c_int32),
                ("dtype", C.c_int32)]


def moments_job(cube, height, width, bands, out, dtype=F32, stride=None, reference=None) -> MomentsJob:
    stride = cube.shape[-1] if stride is None else stride
    return MomentsJob(_ptr(cube), stride, _ptr(out), _ptr(reference), height, width, bands, dtype)


def scene_moments_batch(jobs, workspace=None, stream=None, device="cuda"):
    """Raw moments of many frames (MomentsJob list) with hsi_scene_moments_batch:
    the tensor-path frames run as one launch sequence per element type."""
    torch = _torch()
    arr = (MomentsJob * len(jobs))(*jobs)
    need = lib().hsi_scene_moments_batch_workspace_bytes(arr, len(jobs))
    if workspace is None:
        workspace = torch.empty(max(need, 1), dtype=torch.uint8, device=device)
    check(lib().hsi_scene_moments_batch(arr, len(jobs), _ptr(workspace), workspace.numel(), _stream(stream)),
          "hsi_scene_moments_batch")
    return workspace


def split_moments(m, bands):
    """(sum, outer, count) views of a moments vector."""
    return m[:bands], m[bands:bands + bands * bands].reshape(bands, bands), m[bands + bands * bands]


def statistics_elements(bands, targets) -> int:
    return lib().hsi_statistics_elements(bands, targets)


def unpack_statistics(flat, bands, targets):
    """Packed statistics -> dict (mean, whitener, target_white, target_norm2, cem_weight)."""
    B, T = bands, targets
    o = 0
    out = {}
    for name, n, shape in (("mean", B, (B,)), ("whitener", B * B, (B, B)), ("target_white", T * B, (T, B)),
                           ("target_norm2", T, (T,)), ("cem_weight", T * B, (T, B))):
        out[name] = flat[o:o + n].reshape(shape)
        o += n
    return out


def build_statistics(moments, bands, library=None, loading=1e-6, want64=True, want32=False, cem_weights=None,
                     status=None, library_stride=0, stream=None):
    """FP64 detector statistics on the device for a batch of frames.

    moments: (F, B+B*B+1) or (B+B*B+1,) float64 device tensor.  library: (T, B) shared or
    (F, T, B) per-frame float32 device tensor.  Returns (stats64 (F, n) or None,
    stats32 (F, n) or None, status (F,) int32)."""
    torch = _torch()
    dev = moments.device
    m = moments.reshape(-1, moments_elements(bands))
    F = m.shape[0]
    T = 0 if library is None else library.shape[-2]
    if library is not None and library.dim() == 3:
        library_stride = library.shape[1] * library.shape[2]
    n = statistics_elements(bands, T)
    s64 = torch.zeros((F, n), dtype=torch.float64, device=dev) if want64 else None
    s32 = torch.zeros((F, n), dtype=torch.float32, device=dev) if want32 else None
    if status is None:
        status = torch.full((F,), -1, dtype=torch.int32, device=dev)
    wsb = lib().hsi_factor_workspace_bytes(F, bands)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
    check(lib().hsi_build_statistics(F, bands, T, float(loading), _ptr(m), _ptr(library), library_stride,
                                     _ptr(s64), _ptr(s32), _ptr(cem_weights), _ptr(status), _ptr(ws), wsb,
                                     _stream(stream)), "hsi_build_statistics")
    return s64, s32, status


# ---------------------------------------------------------------------------
# RX / ACE scoring
# ---------------------------------------------------------------------------

def rx_ace(cube, height, width, bands, stats64, num_targets, dtype=F32, stride=None, rx=None, ace_best=None,
           ace_target=None, ace_maps=None, map_stride=None, simt=False, workspace=None, stream=None):
    """RX and ACE maps of one frame from its packed FP64 statistics (build_statistics).
    simt=True runs the plain FP32 CUDA-core path."""
    torch = _torch()
    dev = cube.device
    stride = cube.shape[-1] if stride is None else stride
    P = height * width
    L = lib()
    wsf = L.hsi_rx_ace_simt_workspace_bytes if simt else L.hsi_rx_ace_workspace_bytes
    fn = L.hsi_rx_ace_simt if simt else L.hsi_rx_ace
    if workspace is None:
        workspace = torch.empty(wsf(bands, num_targets), dtype=torch.uint8, device=dev)
    if map_stride is None:
        map_stride = ace_maps.shape[-1] if ace_maps is not None else P
    check(fn(_ptr(cube), height, width, bands, dtype, stride, _ptr(stats64), num_targets, _ptr(rx), _ptr(ace_best),
             _ptr(ace_target), _ptr(ace_maps), map_stride, _ptr(workspace), workspace.numel(), _stream(stream)),
          "hsi_rx_ace")


# ---------------------------------------------------------------------------
# learned screen
# ---------------------------------------------------------------------------

def screen_normaliser(moments, bands, out=None, stream=None):
    """Per-band mean and power-of-two scale (2 * Bp floats) from raw FP64 moments."""
    torch = _torch()
    Bp = (bands + 63) // 64 * 64
    if out is None:
        out = torch.zeros(2 * Bp, device=moments.device)
    check(lib().hsi_screen_normaliser(_ptr(moments), bands, _ptr(out), _stream(stream)), "hsi_screen_normaliser")
    return out


class Screen:
    """Parameters (FP32 master), Adam state and the training / inference calls
    of the learned screen, all through the C ABI."""

    def __init__(self, bands, seed=1, device="cuda"):
        torch = _torch()
        L = lib()
        self.bands = bands
        self.count = int(L.hsi_screen_param_count(bands))
        self.params = torch.zeros(self.count, device=device)
        check(L.hsi_screen_init(_ptr(self.params), bands, seed, None), "hsi_screen_init")
        self.adam = torch.zeros(2 * self.count, device=device)
        self.grads = torch.zeros(self.count, device=device)
        self.loss = torch.zeros(1, device=device)
        self.step = 0
        self._ws = None
        self._buffers = {}

    def _train_buffers(self, batch, device):
        torch = _torch()
        if batch not in self._buffers:
            Bp = (self.bands + 63) // 64 * 64
            wb = lib().hsi_screen_train_workspace_bytes(self.bands, batch)
            self._buffers[batch] = (torch.empty(batch, dtype=torch.int32, device=device),
                                    torch.empty(batch, device=device), torch.empty((Bp, batch), device=device),
                                    torch.empty(wb, dtype=torch.uint8, device=device), wb)
        return self._buffers[batch]

    def train_on(self, cube, height, width, dtype, norm, score, threshold, steps, batch=4096,
                 positive_fraction=0.25, lr=1e-3, pos_weight=2.0, seed=0, capacity=1 << 16, stream=None):
        """`steps` Adam steps on one frame: labels are score >= threshold (the
        plain detector's decision); a quarter of each batch is drawn from its
        positive list, the rest uniformly.  Returns the last loss (device)."""
        L = lib()
        count, pos = detect(score, None, height, width, threshold, 0, HIGHER_IS_BETTER, capacity, stream=stream)
        idx, lab, feats, ws, wb = self._train_buffers(batch, cube.device)
        stride = cube.shape[-1]
        npos = int(batch * positive_fraction)
        s = _stream(stream)
        for k in range(steps):
            check(L.hsi_screen_batch(_ptr(pos), _ptr(count), capacity, height, width, _ptr(score), float(threshold),
                                     (seed << 20) + k, npos, batch, _ptr(idx), _ptr(lab), s), "hsi_screen_batch")
            check(L.hsi_screen_gather(_ptr(cube), dtype, stride, self.bands, _ptr(norm), _ptr(idx), batch,
                                      _ptr(feats), s), "hsi_screen_gather")
            check(L.hsi_screen_gradients(_ptr(self.params), self.bands, _ptr(feats), _ptr(lab), batch,
                                         float(pos_weight), _ptr(self.grads), _ptr(self.loss), _ptr(ws), wb, s),
                  "hsi_screen_gradients")
            self.step += 1
            check(L.hsi_screen_adam(_ptr(self.params), _ptr(self.adam), _ptr(self.grads), self.bands, float(lr),
                                    self.step, s), "hsi_screen_adam")
        return self.loss

    def logits(self, cube, height, width, norm, out=None, stream=None):
        """Logit of every pixel of an fp16 cube (tensor-core inference)."""
        torch = _torch()
        L = lib()
        if out is None:
            out = torch.empty(height * width, device=cube.device)
        if self._ws is None:
            self._ws = torch.empty(L.hsi_screen_infer_workspace_bytes(self.bands), dtype=torch.uint8,
                                   device=cube.device)
        check(L.hsi_screen_infer(_ptr(cube), height, width, self.bands, F16, cube.shape[-1], _ptr(norm),
                                 _ptr(self.params), _ptr(out), _ptr(self._ws), self._ws.numel(), _stream(stream)),
              "hsi_screen_infer")
        return out


def gather_candidates(cube, dtype, bands, width, candidates, count, capacity, out=None, stream=None):
    """Spectra of a candidate list as a compact BSQ cube (bands x capacity, stride = capacity)."""
    torch = _torch()
    if out is None:
        out = torch.empty((bands, capacity), dtype=cube.dtype, device=cube.device)
    check(lib().hsi_gather_candidates(_ptr(cube), dtype, cube.shape[-1], bands, width, _ptr(candidates),
                                      _ptr(count), capacity, _ptr(out), capacity, _stream(stream)),
          "hsi_gather_candidates")
    return out


# ---------------------------------------------------------------------------
# batched frame runner (libhsi_cxx.so, include/hsi_batch.h)
# ---------------------------------------------------------------------------

CXX_LIB_PATH = os.path.join(os.path.dirname(LIB_PATH), "libhsi_cxx.so")
_cxx = None


class BatchFrame(C.Structure):
    _fields_ = [("cube", C.c_void_p), ("raw", C.c_void_p), ("raw_height", C.c_int32), ("raw_width", C.c_int32),
                ("period", C.c_int32), ("height", C.c_int32), ("width", C.c_int32), ("bands", C.c_int32),
                ("dtype", C.c_int32), ("targets", C.c_void_p), ("num_targets", C.c_int32)]


class BatchOptions(C.Structure):
    _fields_ = [("sam_threshold", C.c_float), ("ace_threshold", C.c_float), ("rx_false_alarm_rate", C.c_double),
                ("loading", C.c_double), ("nms_radius", C.c_int32), ("capacity", C.c_int32),
                ("autotune", C.c_int32)]


class BatchOutputs(C.Structure):
    _fields_ = [("sam_best", C.c_void_p), ("sam_target", C.c_void_p), ("rx", C.c_void_p), ("ace_best", C.c_void_p),
                ("ace_target", C.c_void_p), ("detections", C.c_void_p * 3), ("counts", C.c_void_p),
                ("status", C.c_void_p), ("rx_threshold", C.c_float)]


class BatchTuning(C.Structure):
    _fields_ = [("score_ctas_per_sm", C.c_int32), ("tensor_core_rx_frames", C.c_int32),
                ("plain_rx_frames", C.c_int32), ("tuning_ms", C.c_float)]


LAGGED_SAM_CEM = 1
LAGGED_RX_ACE = 2


class LaggedOptions(C.Structure):
    _fields_ = [("height", C.c_int32), ("width", C.c_int32), ("bands", C.c_int32), ("dtype", C.c_int32),
                ("targets", C.c_void_p), ("num_targets", C.c_int32), ("detectors", C.c_int32),
                ("loading", C.c_double), ("sam_threshold", C.c_float), ("cem_threshold", C.c_float),
                ("ace_threshold", C.c_float), ("rx_false_alarm_rate", C.c_double), ("nms_radius", C.c_int32),
                ("capacity", C.c_int32)]


class LaggedOutputs(C.Structure):
    _fields_ = [("frame", C.c_int64), ("statistics_frame", C.c_int64), ("sam_maps", C.c_void_p),
                ("sam_best", C.c_void_p), ("sam_target", C.c_void_p), ("cem_maps", C.c_void_p),
                ("cem_best", C.c_void_p), ("cem_target", C.c_void_p), ("rx", C.c_void_p), ("ace_maps", C.c_void_p),
                ("ace_best", C.c_void_p), ("ace_target", C.c_void_p), ("detections", C.c_void_p * 4),
                ("counts", C.c_void_p), ("status", C.c_void_p), ("map_stride", C.c_int64),
                ("rx_threshold", C.c_float)]


def cxx_lib():
    """libhsi_cxx.so (C++ API and the batch runner's C ABI); raises if not built."""
    global _cxx
    if _cxx is None:
        lib()  # the kernels library first (libhsi_cxx links it)
        if not os.path.exists(CXX_LIB_PATH):
            raise RuntimeError(f"{CXX_LIB_PATH} is missing: build it with `make -C {PKG}`")
        L = C.CDLL(CXX_LIB_PATH)
        vp, i32 = C.c_void_p, C.c_int
        L.hsi_batch_create.argtypes = [C.POINTER(BatchFrame), i32, C.POINTER(BatchOptions), C.POINTER(C.c_int)]
        L.hsi_batch_create.restype = vp
        for name in ("hsi_batch_run", "hsi_batch_capture", "hsi_batch_launch"):
            getattr(L, name).argtypes = [vp, vp]
            getattr(L, name).restype = i32
        L.hsi_batch_outputs_of.argtypes = [vp, i32, C.POINTER(BatchOutputs)]
        L.hsi_batch_outputs_of.restype = i32
        L.hsi_batch_tuning_of.argtypes = [vp, C.POINTER(BatchTuning)]
        L.hsi_batch_tuning_of.restype = i32
        L.hsi_batch_destroy.argtypes = [vp]
        L.hsi_batch_destroy.restype = None
        L.hsi_lagged_create.argtypes = [C.POINTER(LaggedOptions), C.POINTER(C.c_int)]
        L.hsi_lagged_create.restype = vp
        L.hsi_lagged_push.argtypes = [vp, vp, vp]
        L.hsi_lagged_push.restype = i32
        L.hsi_lagged_outputs_of.argtypes = [vp, C.POINTER(LaggedOutputs)]
        L.hsi_lagged_outputs_of.restype = i32
        L.hsi_lagged_destroy.argtypes = [vp]
        L.hsi_lagged_destroy.restype = None
        _cxx = L
    return _cxx


class Batch:
    """A batch of uneven frames run by the library's batched plan.  `frames`:
    dicts with cube (device BSQ tensor at plane_stride) or raw (device mosaic,
    with period), height, width, bands, dtype, targets (numpy T x B float32)."""

    def __init__(self, frames, sam_threshold=0.10, ace_threshold=0.5, rx_false_alarm_rate=1e-3, loading=1e-6,
                 nms_radius=2, capacity=4096, autotune=True):
        import numpy as np
        L = cxx_lib()
        self._keep = []
        arr = (BatchFrame * len(frames))()
        for i, f in enumerate(frames):
            tg = np.ascontiguousarray(f["targets"], np.float32)
            self._keep.append(tg)
            raw = f.get("raw")
            cube = f.get("cube")
            arr[i] = BatchFrame(cube.data_ptr() if cube is not None else None,
                                raw.data_ptr() if raw is not None else None,
                                raw.shape[0] if raw is not None else 0, raw.shape[1] if raw is not None else 0,
                                f.get("period", 0), f.get("height", 0), f.get("width", 0), f["bands"],
                                f.get("dtype", F32), tg.ctypes.data, tg.shape[0])
        opt = BatchOptions(sam_threshold, ace_threshold, rx_false_alarm_rate, loading, nms_radius, capacity,
                           1 if autotune else 0)
        st = C.c_int(0)
        self.handle = L.hsi_batch_create(arr, len(frames), C.byref(opt), C.byref(st))
        check(st.value, "hsi_batch_create")
        self.frames = frames
        self.capacity = capacity

    def run(self, stream=None):
        check(cxx_lib().hsi_batch_run(self.handle, _stream(stream)), "hsi_batch_run")

    def capture(self, stream):
        check(cxx_lib().hsi_batch_capture(self.handle, _stream(stream)), "hsi_batch_capture")

    def launch(self, stream):
        check(cxx_lib().hsi_batch_launch(self.handle, _stream(stream)), "hsi_batch_launch")

    def outputs(self, i):
        o = BatchOutputs()
        check(cxx_lib().hsi_batch_outputs_of(self.handle, i, C.byref(o)), "hsi_batch_outputs_of")
        return o

    def tuning(self):
        t = BatchTuning()
        check(cxx_lib().hsi_batch_tuning_of(self.handle, C.byref(t)), "hsi_batch_tuning_of")
        return {"score_ctas_per_sm": t.score_ctas_per_sm, "tensor_core_rx_frames": t.tensor_core_rx_frames,
                "plain_rx_frames": t.plain_rx_frames, "tuning_ms": round(t.tuning_ms, 2)}

    def close(self):
        if self.handle:
            cxx_lib().hsi_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Lagged:
    """The lagged-statistics video runner (include/hsi_lagged.h): push device
    cubes of one shape in order; frame k is scored with frame k-1's statistics
    while frame k's own are built on an internal stream."""

    def __init__(self, height, width, bands, targets, dtype=F32, detectors=LAGGED_SAM_CEM | LAGGED_RX_ACE,
                 loading=1e-6, sam_threshold=0.10, cem_threshold=0.5, ace_threshold=0.5, rx_false_alarm_rate=1e-3,
                 nms_radius=2, capacity=4096):
        import numpy as np
        L = cxx_lib()
        self._tg = np.ascontiguousarray(targets, np.float32)
        opt = LaggedOptions(height, width, bands, dtype, self._tg.ctypes.data, self._tg.shape[0], detectors, loading,
                            sam_threshold, cem_threshold, ace_threshold, rx_false_alarm_rate, nms_radius, capacity)
        st = C.c_int(0)
        self.handle = L.hsi_lagged_create(C.byref(opt), C.byref(st))
        check(st.value, "hsi_lagged_create")
        self.height, self.width, self.bands, self.targets, self.capacity = height, width, bands, self._tg.shape[0], capacity

    def push(self, cube, stream=None):
        check(cxx_lib().hsi_lagged_push(self.handle, _ptr(cube), _stream(stream)), "hsi_lagged_push")

    def outputs(self):
        o = LaggedOutputs()
        check(cxx_lib().hsi_lagged_outputs_of(self.handle, C.byref(o)), "hsi_lagged_outputs_of")
        return o

    def close(self):
        if self.handle:
            cxx_lib().hsi_lagged_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_copy(ptr, n, dtype, device="cuda"):
    """A new torch tensor holding n elements copied from device memory at `ptr`
    (memory the library owns, e.g. a batch's outputs)."""
    torch = _torch()
    t = torch.empty(n, dtype=dtype, device=device)
    rt = _cudart()
    err = rt.cudaMemcpy(C.c_void_p(t.data_ptr()), C.c_void_p(ptr), t.numel() * t.element_size(), 4)  # Default
    if err != 0:
        raise HsiError(err, "cudaMemcpy")
    return t


_rt = None


def _cudart():
    """The CUDA runtime the library is linked against (already loaded)."""
    global _rt
    if _rt is None:
        lib()
        for name in ("libcudart.so.12", "libcudart.so"):
            try:
                _rt = C.CDLL(name)
                break
            except OSError:
                continue
        if _rt is None:
            raise RuntimeError("the CUDA runtime library is not loadable")
        _rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        _rt.cudaMemcpy.restype = C.c_int
    return _rt
