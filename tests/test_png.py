"""PNG output: the host-side writer (no GPU) and, on the GPU, savePNG of libWR's test
layer (libWR/test/helpers/image.cpp:23-49): the decoded pixels are the ACES bytes of
wrk_tonemap_aces, which are pinned to the reference's own writer by the oracle tests."""
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
