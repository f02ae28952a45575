"""Generates the golden fixtures in this directory from the reference itself.

The reference (trianglestrip/OfflineRenderer) publishes no golden vectors, so the
fixtures come from running the reference's own code where it runs on a CPU: its
shading / sampling / RNG headers (libWR/kernels/*.cuh) and its PNG writer
(libWR/test/helpers/image.cpp), compiled on the host into oracle/_ref/libref.so
by oracle/Makefile from a reference checkout.  Run from the repository root:

    make -C oracle && python tests/golden/make_golden.py

Outputs (small .npz files, committed):
  bsdf_ref.npz     -- 2048 BSDF records (inputs) and the reference's 34 outputs each
  rng_ref.npz      -- PCG hash / uniform for 4096 (seed, dimension) pairs
  cdf_ref.npz      -- light-CDF lower-bound indices for 4096 uniforms on 3 CDFs
  camera_ref.npz   -- camera bases (GLM) for 16 random cameras
  aces_ref.npz     -- the reference PNG writer's bytes for a 64x64 HDR ramp image
  cornell_ref.npz  -- 32x32 Cornell box, 8 spp, rendered by the reference shading
                      code on the host (g++ argument order) with the oracle's CPU
                      traversal: rgb, albedo sum, normal sum and ray counts
"""
from __future__ import annotations

import os
import struct
import sys
import tempfile
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from offlinerenderer_b200 import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def read_png_rgb8(path: str) -> np.ndarray:
    """Minimal PNG reader for 8-bit RGB, non-interlaced (what stb_image_write emits)."""
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = 0
    while pos < len(data):
        ln, typ = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + ln]
        if typ == b"IHDR":
            w, h, bd, ct, _, _, il = struct.unpack(">IIBBBBB", body)
            assert bd == 8 and ct == 2 and il == 0
        elif typ == b"IDAT":
            idat += body
        pos += 12 + ln
    raw = zlib.decompress(idat)
    stride = 3 * w
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    p = 0
    for y in range(h):
        f = raw[p]
        line = np.frombuffer(raw[p + 1:p + 1 + stride], np.uint8).astype(np.int32)
        p += 1 + stride
        cur = np.zeros(stride, np.int32)
        for x in range(stride):
            a = cur[x - 3] if x >= 3 else 0
            b = prev[x]
            c = prev[x - 3] if x >= 3 else 0
            if f == 0:
                v = line[x]
            elif f == 1:
                v = line[x] + a
            elif f == 2:
                v = line[x] + b
            elif f == 3:
                v = line[x] + ((a + b) >> 1)
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                pr = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                v = line[x] + pr
            cur[x] = v & 0xFF
        out[y] = cur
        prev = cur
    return out.reshape(h, w, 3)


def main() -> None:
    ref = pyoracle.Reference()
    inp = pyoracle.random_bsdf_inputs(2048, seed=12345)
    np.savez_compressed(os.path.join(OUT, "bsdf_ref.npz"), inputs=inp, outputs=ref.bsdf(inp))

    rng = np.random.default_rng(7)
    seeds = rng.integers(0, 2 ** 32, 4096, dtype=np.uint64).astype(np.uint32)
    dims = rng.integers(0, 64, 4096).astype(np.uint32)
    h, u = ref.rng(seeds, dims)
    np.savez_compressed(os.path.join(OUT, "rng_ref.npz"), seeds=seeds, dims=dims, hash=h, u=u)

    cdfs, us, idx = [], [], []
    for n in (1, 2, 64):
        w = rng.uniform(0.1, 3.0, n).astype(np.float32)
        cdf = (np.cumsum(w, dtype=np.float32) / np.float32(w.sum(dtype=np.float32))).astype(np.float32)
        uu = rng.random(4096).astype(np.float32)
        uu[:8] = [0.0, 1.0, cdf[0], cdf[-1], np.nextafter(cdf[0], 0), np.nextafter(cdf[0], 2), 0.5, 0.999999]
        cdfs.append(np.pad(cdf, (0, 64 - n)))
        us.append(uu)
        idx.append(ref.cdf_sample(cdf, uu))
    np.savez_compressed(os.path.join(OUT, "cdf_ref.npz"), cdf=np.array(cdfs), n=np.array([1, 2, 64]), u=np.array(us),
                        index=np.array(idx))

    cams, bases = [], []
    for _ in range(16):
        c = scenes.Camera(position=tuple(rng.uniform(-3, 3, 3)), target=tuple(rng.uniform(-1, 1, 3)),
                          up=(0.0, 1.0, 0.0), fovY=float(rng.uniform(0.3, 1.4)))
        cams.append(list(c.position) + list(c.target) + list(c.up) + [c.fovY])
        bases.append(ref.camera_basis(c))
    np.savez_compressed(os.path.join(OUT, "camera_ref.npz"), cameras=np.array(cams, np.float32),
                        basis=np.array(bases, np.float32))

    y, x = np.mgrid[0:64, 0:64].astype(np.float32)
    img = np.stack([x / 16.0, y / 20.0, (x * y) / 700.0], -1).astype(np.float32)
    img[0, :3] = [0.0, 1e-6, 100.0]
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ramp.png")
        ref.save_png(p, img)
        png = read_png_rgb8(p)
    np.savez_compressed(os.path.join(OUT, "aces_ref.npz"), rgb=img, bytes=png)

    sd = scenes.cornell(32, 32, 8, seed=0)
    rs = ref.scene(sd)
    rgb, alb, nrm, st = rs.render()
    np.savez_compressed(os.path.join(OUT, "cornell_ref.npz"), rgb=rgb, albedo=alb, normal=nrm,
                        extension_rays=st["extension_rays"], shadow_rays=st["shadow_rays"])
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
