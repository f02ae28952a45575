"""Image output.  PNG: the host-side writer (no GPU) and, on the GPU, savePNG of
libWR's test layer (libWR/test/helpers/image.cpp:23-49): the decoded pixels are the
ACES bytes of wrk_tonemap_aces, which are pinned to the reference's own writer by the
oracle tests.  OpenEXR and Radiance RGBE outputs of the linear radiance: read back
with independent readers written from the file-format specifications."""
import struct
import zlib

import numpy as np
import pytest


def _decode_png(path):
    d = open(path, "rb").read()
    assert d[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = None
    while pos < len(d):
        n, = struct.unpack(">I", d[pos:pos + 4])
        typ, body = d[pos + 4:pos + 8], d[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", d[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(typ + body)
        if typ == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and ctype == 2
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(h, w, 3)


def test_png_writer_round_trip(wrk_lib, tmp_path):
    rng = np.random.default_rng(5)
    img = rng.integers(0, 256, (37, 53, 3), dtype=np.uint8)
    p = tmp_path / "x.png"
    assert wrk_lib.lib().wrk_png_write(str(p).encode(), np.ascontiguousarray(img).ctypes.data, 53, 37) == 0
    assert np.array_equal(_decode_png(p), img)
    assert wrk_lib.lib().wrk_png_write(str(p).encode(), None, 53, 37) != 0


@pytest.mark.gpu
def test_save_png_is_the_aces_image(gpu, tmp_path):
    from offlinerenderer_b200 import scenes

    sd = scenes.cornell(64, 48, 4, seed=1)
    res = gpu.Renderer(capacity=1 << 14).render(gpu.Scene.from_data(sd))
    p = tmp_path / "cornell.png"
    gpu.save_png(str(p), res.rgb)
    assert np.array_equal(_decode_png(p), gpu.tonemap_aces(res.rgb))


# ---- HDR outputs (OpenEXR, Radiance RGBE): independent readers of the formats ----
def _read_exr(path):
    d = open(path, "rb").read()
    assert d[:4] == b"\x76\x2f\x31\x01" and struct.unpack("<I", d[4:8])[0] == 2
    pos, attrs = 8, {}
    while d[pos] != 0:
        e = d.index(b"\0", pos)
        name = d[pos:e].decode()
        e2 = d.index(b"\0", e + 1)
        typ = d[e + 1:e2].decode()
        size, = struct.unpack("<i", d[e2 + 1:e2 + 5])
        attrs[name] = (typ, d[e2 + 5:e2 + 5 + size])
        pos = e2 + 5 + size
    pos += 1
    for req in ("channels", "compression", "dataWindow", "displayWindow", "lineOrder", "pixelAspectRatio",
                "screenWindowCenter", "screenWindowWidth"):
        assert req in attrs, req
    assert attrs["compression"] == ("compression", b"\0")
    x0, y0, x1, y1 = struct.unpack("<4i", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    ch, p, chans = attrs["channels"][1], 0, []
    while ch[p] != 0:
        e = ch.index(b"\0", p)
        name = ch[p:e].decode()
        ptype, = struct.unpack("<i", ch[e + 1:e + 5])
        xs, ys = struct.unpack("<2i", ch[e + 9:e + 17])
        chans.append((name, ptype, xs, ys))
        p = e + 17
    assert [c[0] for c in chans] == sorted(c[0] for c in chans)
    offs = struct.unpack(f"<{h}Q", d[pos:pos + 8 * h])
    planes = {c[0]: np.zeros((h, w), np.float32) for c in chans}
    for off in offs:
        y, n = struct.unpack("<iI", d[off:off + 8])
        row = np.frombuffer(d[off + 8:off + 8 + n], "<f4").reshape(len(chans), w)
        for k, c in enumerate(chans):
            assert c[1] == 2 and c[2] == 1 and c[3] == 1
            planes[c[0]][y] = row[k]
    return np.stack([planes["R"], planes["G"], planes["B"]], -1)


def _read_hdr(path):
    d = open(path, "rb").read()
    head, rest = d.split(b"\n\n", 1)
    assert head.startswith(b"#?RADIANCE") and b"FORMAT=32-bit_rle_rgbe" in head
    line, rest = rest.split(b"\n", 1)
    _, h, _, w = line.split()
    h, w = int(h), int(w)
    out, pos = np.zeros((h, w, 4), np.uint8), 0
    for y in range(h):
        if rest[pos] == 2 and rest[pos + 1] == 2 and (rest[pos + 2] << 8 | rest[pos + 3]) == w:
            pos += 4
            for c in range(4):
                x = 0
                while x < w:
                    n = rest[pos]
                    pos += 1
                    if n > 128:  # a run of one byte
                        out[y, x:x + n - 128, c] = rest[pos]
                        pos += 1
                        x += n - 128
                    else:
                        out[y, x:x + n, c] = np.frombuffer(rest[pos:pos + n], np.uint8)
                        pos += n
                        x += n
        else:
            out[y] = np.frombuffer(rest[pos:pos + 4 * w], np.uint8).reshape(w, 4)
            pos += 4 * w
    assert pos == len(rest)
    return out


def _rgbe_np(img):
    """Ward's RGBE encoding, restated with numpy (float32 arithmetic)."""
    img = img.astype(np.float32)
    v = img.max(-1)
    live = v >= 1e-32  # False for NaN too
    img = np.where(live[..., None], img, 0).astype(np.float32)
    v = np.where(live, v, 1).astype(np.float32)
    m, e = np.frexp(v)
    scale = (m.astype(np.float32) * np.float32(256.0) / v).astype(np.float32)
    q = np.clip(img * scale[..., None], 0, None).astype(np.uint8)
    out = np.concatenate([q, (e + 128).astype(np.uint8)[..., None]], -1)
    out[~live] = 0
    return out


@pytest.mark.parametrize("hw", [(37, 53), (5, 7), (1, 1)])
def test_exr_writer_round_trip(wrk_lib, tmp_path, hw):
    rng = np.random.default_rng(11)
    img = (rng.gamma(0.5, 2.0, hw + (3,)) * rng.choice([1e-3, 1.0, 1e3], hw + (1,))).astype(np.float32)
    img[0, 0] = [0.0, -1.5, 65504.0 * 4]
    p = tmp_path / "x.exr"
    wrk_lib.save_exr(str(p), img)
    assert np.array_equal(_read_exr(p), img)


@pytest.mark.parametrize("hw", [(19, 40), (3, 5)])
def test_hdr_writer_matches_rgbe(wrk_lib, tmp_path, hw):
    rng = np.random.default_rng(12)
    img = (rng.gamma(0.5, 2.0, hw + (3,)) * rng.choice([1e-3, 1.0, 1e3], hw + (1,))).astype(np.float32)
    img[0, 0] = [0.0, 0.0, 0.0]
    img[0, 1] = [np.nan, 1.0, 1.0]
    p = tmp_path / "x.hdr"
    wrk_lib.save_hdr(str(p), img)
    got = _read_hdr(p)
    assert np.array_equal(got, _rgbe_np(img))
    dec = got[..., :3].astype(np.float64) * np.ldexp(1.0, got[..., 3:].astype(np.int64) - 136)
    ok = np.isfinite(img).all(-1) & (img.max(-1) > 1e-30)
    assert np.allclose(dec[ok], img[ok], rtol=1.0 / 128, atol=img[ok].max(-1, keepdims=True) / 128)


def test_hdr_exr_reject_bad_arguments(wrk_lib, tmp_path):
    L = wrk_lib.lib()
    assert L.wrk_exr_write(str(tmp_path / "a.exr").encode(), None, 4, 4) != 0
    assert L.wrk_hdr_write(str(tmp_path / "a.hdr").encode(), None, 4, 4) != 0
    buf = np.zeros(12, np.float32)
    assert L.wrk_exr_write(str(tmp_path / "a.exr").encode(), buf.ctypes.data, 0, 4) != 0
    assert L.wrk_hdr_write(b"/nonexistent-dir/x.hdr", buf.ctypes.data, 2, 2) != 0


def test_cpp_save_exr_hdr(wrk_lib, tmp_path):
    """test_helpers::saveEXR / saveHDR through the C++ API (host-only writers)."""
    import os
    import subprocess

    from conftest import ROOT

    exe = tmp_path / "save_hdr"
    lib_dir = os.path.dirname(wrk_lib.LIB_PATH)
    subprocess.run(["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "save_hdr.cpp"), "-o", str(exe), "-L", lib_dir, "-lwrk",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    r = subprocess.run([str(exe), str(tmp_path / "g.exr"), str(tmp_path / "g.hdr")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "saveEXR" in r.stdout, r.stdout + r.stderr
    y, x = np.mgrid[0:10, 0:24].astype(np.float32)
    img = np.stack([np.float32(0.25) * x, np.float32(0.5) * y + np.float32(0.125),
                    np.float32(100.0) / (1 + x + y)], -1).astype(np.float32)
    assert np.array_equal(_read_exr(tmp_path / "g.exr"), img)
    assert np.array_equal(_read_hdr(tmp_path / "g.hdr"), _rgbe_np(img))
