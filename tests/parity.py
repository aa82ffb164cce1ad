"""Helpers for the end-to-end detection-set parity tests (not a test module).

Detection-set parity rule.  The reference does not define one for a GPU path
whose scores differ from its own in the last bits, so it is stated here: the
GPU's detection index set must equal the reference CPU scorer's
(src/sam_cpu.cpp:116-138 detect_cpu, over sam_best_cpu / cem_best_cpu /
ace_best_cpu scores) for every pixel p except those where
  * |s_ref(p) - threshold| <= tol  (the two scores may straddle the threshold),
  * or some neighbour q in p's NMS window has |s_ref(q) - s_ref(p)| <= tol
    (the NMS order of p and q may flip).
With nms_radius 0 only the first clause applies.  `tol` is stated per test and
bounds |s_gpu - s_ref| (checked in the test from both arms' error against the
FP64 oracle).
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

THREADS = max(1, min(16, os.cpu_count() or 1))


def excluded(ref_score, height, width, threshold, radius, tol, rel=False):
    """Boolean (H, W) mask of the pixels the parity rule leaves out.  With
    rel, the tolerance at a score s is tol * max(1, |s|)."""
    s = np.asarray(ref_score, np.float64).reshape(height, width)
    band = tol * np.maximum(1.0, np.abs(s)) if rel else tol
    ex = np.abs(s - threshold) <= (tol * max(1.0, abs(threshold)) if rel else tol)
    if radius > 0:
        pad = np.pad(s, radius, constant_values=np.nan)
        for dy in range(-radius, radius + 1):
            for dx in range(-radius, radius + 1):
                if dy == 0 and dx == 0:
                    continue
                q = pad[radius + dy:radius + dy + height, radius + dx:radius + dx + width]
                with np.errstate(invalid="ignore"):
                    ex |= np.abs(q - s) <= band
    return ex


def index_set(dets, width):
    """Linear indices (y * width + x) of a detection record array."""
    return dets["y"].astype(np.int64) * width + dets["x"].astype(np.int64)


def gpu_records(hsi, count, out, capacity):
    """The GPU list as a record array (x, y, target, score); it must fit the capacity."""
    n, rec = hsi.detections_to_numpy(count, out, capacity)
    assert n <= capacity, f"{n} detections overflow the test's capacity {capacity}"
    return rec


def compare_lists(gpu, ref, ref_score, height, width, threshold, radius, tol, margin=None, rel=False):
    """Check the parity rule; returns a summary dict.

    gpu, ref: record arrays (raster order).  margin: optional (P,) FP64 gap
    between the best and the second-best target of each pixel; where it is
    <= tol the best-target ids may differ.  rel: the tolerance at a score s
    is tol * max(1, |s|) (responses without a fixed scale, such as CEM)."""
    ex = excluded(ref_score, height, width, threshold, radius, tol, rel).reshape(-1)
    gi, ri = index_set(gpu, width), index_set(ref, width)
    assert np.all(np.diff(gi) > 0), "GPU list is not in raster order"
    gs, rs = set(gi.tolist()), set(ri.tolist())
    diff = np.array(sorted(gs ^ rs), dtype=np.int64)
    bad = diff[~ex[diff]] if diff.size else diff
    assert bad.size == 0, (f"{bad.size} pixels outside the tolerance band differ between the lists, "
                           f"first {bad[:8].tolist()}")
    # records of the pixels in both lists
    common, g_at, r_at = np.intersect1d(gi, ri, return_indices=True)
    rs_ = ref["score"][r_at].astype(np.float64)
    ds = np.abs(gpu["score"][g_at].astype(np.float64) - rs_)
    bound = tol * np.maximum(1.0, np.abs(rs_)) if rel else np.full(ds.shape, tol)
    assert ds.size == 0 or np.all(ds <= bound), f"detection scores differ by up to {ds.max():.3e}"
    idiff = gpu["target"][g_at] != ref["target"][r_at]
    if margin is not None and idiff.any():
        m = np.asarray(margin)[common[idiff]]
        assert np.all(m <= bound[idiff]), "best-target ids differ where the two best targets are not tied"
    elif margin is None:
        assert not idiff.any(), "best-target ids differ"
    union = np.array(sorted(gs | rs), dtype=np.int64)
    return {"gpu": len(gs), "ref": len(rs), "common": int(common.size), "differ": int(diff.size),
            "excluded_in_union": int(ex[union].sum()) if union.size else 0, "id_ties": int(idiff.sum())}


def best_margin(maps, higher_is_better):
    """Gap between the best and the second-best per-target value, per pixel."""
    m = np.asarray(maps, np.float64)
    if m.shape[0] < 2:
        return np.full(m.shape[1], np.inf)
    part = np.sort(m, axis=0)
    return (part[-1] - part[-2]) if higher_is_better else (part[1] - part[0])


def chunks(n, parts):
    step = (n + parts - 1) // parts
    return [(a, min(n, a + step)) for a in range(0, n, step)]


def fp64_moments_parallel(orc, host):
    """FP64 oracle moments of a (B, P) cube, summed over pixel chunks in threads."""
    import ctypes as C
    lib = orc.fp64_lib()
    B, P = host.shape
    host = np.ascontiguousarray(host, np.float32)
    parts = chunks(P, THREADS)
    sums = [np.zeros(B) for _ in parts]
    outs = [np.zeros((B, B)) for _ in parts]
    base = host.ctypes.data

    def run(k):
        a, b = parts[k]
        lib.orc_moments(C.cast(base + 4 * a, C.POINTER(C.c_float)), b - a, P, B,
                        sums[k].ctypes.data_as(C.POINTER(C.c_double)), outs[k].ctypes.data_as(C.POINTER(C.c_double)))

    with ThreadPoolExecutor(len(parts)) as ex:
        list(ex.map(run, range(len(parts))))
    return sum(sums), sum(outs), float(P)


def fp64_ace_parallel(orc, host, S):
    """FP64 oracle ACE (best, target, rx, per-target maps) over pixel chunks in threads."""
    import ctypes as C
    lib = orc.fp64_lib()
    B, P = host.shape
    T = S["target_norm2"].shape[0]
    host = np.ascontiguousarray(host, np.float32)
    score = np.empty(P, np.float32)
    which = np.empty(P, np.int32)
    rxm = np.empty(P, np.float32)
    allm = np.empty((T, P), np.float32)
    d = {k: np.ascontiguousarray(S[k], np.float64) for k in ("mean", "whitener", "target_white", "target_norm2")}
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    parts = chunks(P, THREADS)

    def run(k):
        a, b = parts[k]
        n = b - a
        tmp = np.empty((T, n), np.float32)
        lib.orc_ace(C.cast(host.ctypes.data + 4 * a, C.POINTER(C.c_float)), n, P, B, fp(d["mean"]),
                    fp(d["whitener"]), fp(d["target_white"]), fp(d["target_norm2"]), T,
                    C.cast(score.ctypes.data + 4 * a, C.POINTER(C.c_float)),
                    C.cast(which.ctypes.data + 4 * a, C.POINTER(C.c_int32)),
                    C.cast(rxm.ctypes.data + 4 * a, C.POINTER(C.c_float)),
                    tmp.ctypes.data_as(C.POINTER(C.c_float)))
        allm[:, a:b] = tmp

    with ThreadPoolExecutor(len(parts)) as ex:
        list(ex.map(run, range(len(parts))))
    return score, which, rxm, allm


def ref_rows_parallel(fn, cube, *args):
    """Run a per-pixel reference scorer (ref_sam_best, ref_ace_best, ref_cem_best)
    over row bands of a (B, H, W) cube in threads and stitch the outputs.
    Each pixel's arithmetic is the reference's own; only the rows a call sees
    differ."""
    B, H, W = cube.shape
    parts = chunks(H, THREADS)

    def run(k):
        a, b = parts[k]
        return fn(np.ascontiguousarray(cube[:, a:b, :]), *args)

    with ThreadPoolExecutor(len(parts)) as ex:
        res = list(ex.map(run, range(len(parts))))
    assert all(r is not None for r in res), "the reference scorer failed"
    return tuple(np.concatenate([r[i] for r in res]) for i in range(len(res[0])))
