"""ENVI reading (include/hsi/envi.hpp) against the reference's own read_envi.

Both readers run here on the CPU: the reference's compiled from its sources
(oracle/_ref, ref_read_envi) and this library's (tests/cpp/envi_dump). Every
sample type in both byte orders and all three interleaves, header offsets, data
file names, comment lines, wrapped and non-numeric wavelength lists, and the
error cases must give the same floats (bit for bit) or the same message.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "hsi-detectors-cuda_b200")
DUMP = os.path.join(PKG, "build", "tests", "envi_dump")

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")

DTYPES = {1: "u1", 2: "i2", 3: "i4", 4: "f4", 5: "f8", 12: "u2", 13: "u4"}


@pytest.fixture(scope="module", autouse=True)
def _built():
    subprocess.run(["make", "-s", "-j8", "-C", PKG, "all", "tests"], check=True, capture_output=True, text=True)


def _ours(hdr, to, tmp_path):
    out = str(tmp_path / "dump.bin")
    r = subprocess.run([DUMP, hdr, str(to), out], capture_output=True, text=True, timeout=60)
    if r.returncode == 3:
        raise RuntimeError(r.stderr.strip()[len("error: "):])
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, np.uint8)
    dims = raw[:16].view(np.int32)
    n = int(dims[0]) * int(dims[1]) * int(dims[2])
    data = raw[16:16 + 4 * n].view(np.float32)
    wl = raw[16 + 4 * n:].view(np.float32)
    assert wl.size == dims[3]
    return (int(dims[0]), int(dims[1]), int(dims[2])), data, wl


def _same(hdr, to, tmp_path):
    shape, data, wl = oracle.ref_read_envi(hdr, to)
    shape2, data2, wl2 = _ours(hdr, to, tmp_path)
    assert shape2 == shape
    assert np.array_equal(data2.view(np.uint32), data.view(np.uint32))
    assert np.array_equal(wl2.view(np.uint32), wl.view(np.uint32))
    return shape, data, wl


def _write(tmp_path, name, header, payload, data_name=None):
    hdr = tmp_path / name
    hdr.write_text(header)
    stem = name[:-4] if name.lower().endswith(".hdr") else name
    (tmp_path / (data_name if data_name is not None else stem)).write_bytes(payload)
    return str(hdr)


def _samples(rng, code, n):
    dt = np.dtype(DTYPES[code])
    if dt.kind == "f":
        return (rng.standard_normal(n) * 3).astype(dt)
    info = np.iinfo(dt)
    v = rng.integers(info.min, info.max, n, dtype=np.int64, endpoint=True)
    v[:4] = [info.min, info.max, 0, 1]
    return v.astype(dt)


@pytest.mark.parametrize("code", sorted(DTYPES))
@pytest.mark.parametrize("big", [False, True])
@pytest.mark.parametrize("interleave", ["bsq", "bil", "bip"])
def test_every_type_order_and_interleave_reads_as_the_reference(tmp_path, code, big, interleave):
    H, W, B = 5, 7, 3
    rng = np.random.default_rng(code * 10 + big)
    s = _samples(rng, code, H * W * B)
    payload = s.astype(s.dtype.newbyteorder(">" if big else "<")).tobytes()
    header = (f"ENVI\nsamples = {W}\nlines = {H}\nbands = {B}\ndata type = {code}\n"
              f"interleave = {interleave}\nbyte order = {1 if big else 0}\n")
    hdr = _write(tmp_path, "cube.hdr", header, payload)
    for to in (0, 1, 2):
        shape, _, _ = _same(hdr, to, tmp_path)
        assert shape == (H, W, B)


def test_header_offset_names_comments_and_wavelengths(tmp_path):
    H, W, B = 4, 6, 5
    rng = np.random.default_rng(3)
    s = rng.standard_normal(H * W * B).astype("<f4")
    header = ("ENVI\n; licence: see https://example.org/a=b\n"
              f"Samples = {W}\nLINES   =   {H}\nbands = {B}\nData Type = 4\n"
              "header offset = 37\ninterleave = BIP\n"
              "wavelength = {\n  400.5, 410.25,\n  420.0, 430.0,\n 440.0 }\n"
              "description = {a wrapped\n description}\n")
    hdr = _write(tmp_path, "scene.HDR", header, b"\x07" * 37 + s.tobytes(), data_name="scene.img")
    shape, _, wl = _same(hdr, 0, tmp_path)
    assert shape == (H, W, B)
    assert np.array_equal(wl, np.array([400.5, 410.25, 420.0, 430.0, 440.0], np.float32))
    # a wavelength list that is not numeric is dropped
    hdr2 = _write(tmp_path, "named.hdr", header.replace("400.5", "band one"), b"\x07" * 37 + s.tobytes(),
                  data_name="named.dat")
    _, _, wl2 = _same(hdr2, 0, tmp_path)
    assert wl2.size == 0


@pytest.mark.parametrize("header, payload_bytes, message", [
    ("samples = 2\nlines = 2\ndata type = 4\n", 64, "missing required field 'bands'"),
    ("samples = two\nlines = 2\nbands = 1\ndata type = 4\n", 64, "is not an integer"),
    ("samples = 2\nlines = 2\nbands = 1\ndata type = 4\nwavelength = {1, 2\n", 64, "unterminated '{'"),
    ("samples = 2\nlines = 2\nbands = 1\ndata type = 4\ninterleave = bsx\n", 64, "unknown ENVI interleave"),
    ("samples = 2\nlines = 2\nbands = 1\ndata type = 6\n", 64, "unsupported ENVI data type 6"),
    ("samples = 2\nlines = 2\nbands = 2\ndata type = 4\n", 12, "bytes, need 32"),
])
def test_errors_match_the_reference(tmp_path, header, payload_bytes, message):
    hdr = _write(tmp_path, "bad.hdr", header, b"\0" * payload_bytes)
    with pytest.raises(RuntimeError) as ref:
        oracle.ref_read_envi(hdr, 0)
    with pytest.raises(RuntimeError) as ours:
        _ours(hdr, 0, tmp_path)
    assert message in str(ref.value)
    assert str(ours.value) == str(ref.value)


def test_missing_data_file_matches_the_reference(tmp_path):
    hdr = tmp_path / "lonely.hdr"
    hdr.write_text("samples = 2\nlines = 2\nbands = 1\ndata type = 4\n")
    with pytest.raises(RuntimeError) as ref:
        oracle.ref_read_envi(str(hdr), 0)
    with pytest.raises(RuntimeError) as ours:
        _ours(str(hdr), 0, tmp_path)
    assert "no ENVI data file found" in str(ref.value)
    assert str(ours.value) == str(ref.value)
